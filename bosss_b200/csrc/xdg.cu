// xdg.cu -- XDG bulk evaluation with moment-fitted cut-cell rules.
//
// Reference counterparts:
//  * XEvaluatorNonlin.Evaluate, per-species bulk part (XSpatialOperatorMk2_XEvaluators.cs:372-511,
//    SpeciesBulkEval per species :409-430): each species s evaluates its bulk operator (here
//    XLaplace_Bulk = SIPLaplace with nu = mu_s, XLaplace.cs:50-120) on the cells and faces that
//    contain s, with species-restricted quadrature on cut cells;
//  * cut-cell volume and face rules by moment fitting (LevelSetComboRuleFactory2.cs:300-528):
//    candidate nodes, moments b_m = int_{K cap s} phi_m, min-norm least squares
//    w = argmin |w| s.t. Phi w = b (IMatrixExtensions.cs:2318-2340, LAPACK DGELSY).
//
// Split of the work: the uncut cells and faces of a species go through the tensor kernel with
// species masks (EvalArgs::vol_flag / face_flag); the cut cells and cut faces go through
// the explicit-rule kernel below, which adds its contributions with atomics. Moments are
// integrated on the device by two-level uniform subdivision of the cell (or face) with
// tensor Gauss rules per sub-box (exact on uncut sub-boxes); the weights are solved on the
// device in FP64 per rule (Gram matrix, Cholesky, degree reduced on loss of rank).
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <string>
#include <functional>
#include <vector>

#include "handle.h"

namespace bosss {

constexpr int XDG_MAXM = 35;     // moments of degree <= 4 in 3D
constexpr int XDG_MAXN = 128;    // nodes per rule

struct LevelSetDev {
    int type;
    double c[3];
    double r;
};

__host__ __device__ inline double ls_phi(const LevelSetDev& L, const double* x) {
    const double a = x[0] - L.c[0], b = x[1] - L.c[1], c = x[2] - L.c[2];
    return sqrt(a * a + b * b + c * c) - L.r;
}

// sign classification of an axis-aligned box [lo, hi] for the sphere:
// -1 fully inside (phi < 0), +1 fully outside, 0 cut
__host__ __device__ inline int ls_box(const LevelSetDev& L, const double* lo, const double* hi, int dim_mask) {
    double dmin2 = 0.0, dmax2 = 0.0;
    for (int d = 0; d < 3; ++d) {
        if (!(dim_mask & (1 << d))) {   // degenerate direction (face): lo == hi
            const double v = lo[d] - L.c[d];
            dmin2 += v * v;
            dmax2 += v * v;
            continue;
        }
        const double cl = fmin(fmax(L.c[d], lo[d]), hi[d]) - L.c[d];
        dmin2 += cl * cl;
        const double f = fmax(fabs(lo[d] - L.c[d]), fabs(hi[d] - L.c[d]));
        dmax2 += f * f;
    }
    if (sqrt(dmax2) <= L.r) return -1;
    if (sqrt(dmin2) >= L.r) return +1;
    return 0;
}

__host__ __device__ inline int nmodes3(int p) { return (p + 1) * (p + 2) * (p + 3) / 6; }
__host__ __device__ inline int nmodes2(int p) { return (p + 1) * (p + 2) / 2; }

__host__ __device__ inline void legendre_vals(int K, double x, double* L, double* dL) {
    double P0 = 1.0, P1 = x, dP0 = 0.0, dP1 = 1.0;
    double P[5], dP[5];
    P[0] = 1.0;
    dP[0] = 0.0;
    if (K >= 1) {
        P[1] = x;
        dP[1] = 1.0;
    }
    for (int m = 1; m < K; ++m) {
        const double P2 = ((2 * m + 1) * x * P1 - m * P0) / (m + 1);
        const double dP2 = dP0 + (2 * m + 1) * P1;
        P[m + 1] = P2;
        dP[m + 1] = dP2;
        P0 = P1;
        P1 = P2;
        dP0 = dP1;
        dP1 = dP2;
    }
    for (int a = 0; a <= K; ++a) {
        const double s = sqrt((2.0 * a + 1.0) / 2.0);
        L[a] = s * P[a];
        if (dL) dL[a] = s * dP[a];
    }
}

// reference basis (3D, reference order) values at xi: out[n], n < nmodes3(p)
__host__ __device__ inline void basis3(int p, const double* xi, double* out) {
    double Lx[5], Ly[5], Lz[5];
    legendre_vals(p, xi[0], Lx, nullptr);
    legendre_vals(p, xi[1], Ly, nullptr);
    legendre_vals(p, xi[2], Lz, nullptr);
    int n = 0;
    for (int deg = 0; deg <= p; ++deg)
        for (int a = 0; a <= deg; ++a)
            for (int b = 0; b <= deg - a; ++b) out[n++] = Lx[a] * Ly[b] * Lz[deg - a - b];
}

__host__ __device__ inline void basis2(int p, const double* t, double* out) {
    double L1[5], L2[5];
    legendre_vals(p, t[0], L1, nullptr);
    legendre_vals(p, t[1], L2, nullptr);
    int n = 0;
    for (int deg = 0; deg <= p; ++deg)
        for (int a = 0; a <= deg; ++a) out[n++] = L1[a] * L2[deg - a];
}

// Gauss-Legendre nodes/weights (host), ascending
static void gauss(int n, std::vector<double>& x, std::vector<double>& w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    const long double PI = 3.141592653589793238462643383279502884L;
    for (int i = 0; i < n; ++i) {
        long double z = std::cos(PI * (i + 0.75L) / (n + 0.5L)), dp = 1.0L;
        for (int it = 0; it < 80; ++it) {
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
            if (std::fabs((double)dz) < 1e-19) break;
        }
        long double p0 = 1.0L, p1 = z;
        for (int m = 1; m < n; ++m) {
            long double p2 = ((2 * m + 1) * z * p1 - m * p0) / (m + 1);
            p0 = p1;
            p1 = p2;
        }
        long double pn = (n == 1) ? z : p1, pm = (n == 1) ? 1.0L : p0;
        dp = n * (z * pn - pm) / (z * z - 1.0L);
        x[n - 1 - i] = (double)z;
        w[n - 1 - i] = (double)(2.0L / ((1.0L - z * z) * dp * dp));
    }
    if (n % 2 == 1) x[n / 2] = 0.0;
}

// ------------------------------------------------------------------ device: moments
// One rule item: a cut cell (dim 3) or a cut face (dim 2: in-plane dims t1 < t2, fixed
// coordinate along `dir` at `xfix`) restricted to species `sp` (-1 inside, +1 outside).
struct CutItem {
    long long cell;     // cell (volume) / lower or own cell (face)
    int dim;            // 3 volume, 2 face
    int dir;            // face normal direction
    int side;           // face: 0 lower, 1 upper face of `cell`
    int sp;             // -1 species A (phi < 0), +1 species B
    int p;              // moment degree requested
    int nnodes;
    long long node_off; // offset into the node / weight arrays
    double center[3];   // cell centre (volume) or face centre (face)
    double h[3];
};

struct Sub {
    int S1, S2;   // coarse and fine subdivision per direction
    double gx[3], gw[3];   // 3-point Gauss rule on [-1,1]
};

// The moment degree and the dimension are template parameters, so the accumulators and the
// basis values at a node stay in registers.
template <int PD, int DIMS>
__device__ __forceinline__ void moments_item(const CutItem& it, long long r, const LevelSetDev& L, const Sub& sub,
                                             double* __restrict__ mom, int* cutlist, int& ncut,
                                             double (*red)[33]) {
    constexpr int M = (DIMS == 3) ? (PD + 1) * (PD + 2) * (PD + 3) / 6 : (PD + 1) * (PD + 2) / 2;
    double acc[M];
#pragma unroll
    for (int m = 0; m < M; ++m) acc[m] = 0.0;
    constexpr int dims = DIMS;
    int t[3];   // reference directions integrated
    if (dims == 3) {
        t[0] = 0;
        t[1] = 1;
        t[2] = 2;
    } else {
        t[0] = (it.dir == 0) ? 1 : 0;
        t[1] = (it.dir == 2) ? 1 : 2;
    }
    const int S1 = sub.S1, S2 = sub.S2;
    const long long ncoarse = (dims == 3) ? (long long)S1 * S1 * S1 : (long long)S1 * S1;
    const long long nfine = (dims == 3) ? (long long)S2 * S2 * S2 : (long long)S2 * S2;
    auto to_phys = [&](const double* rr, double* x) {
        for (int d = 0; d < 3; ++d) x[d] = it.center[d];
        for (int k = 0; k < dims; ++k) x[t[k]] = it.center[t[k]] + 0.5 * it.h[t[k]] * rr[k];
    };
    auto classify = [&](const double* a, const double* b) {
        double plo[3], phi_[3];
        to_phys(a, plo);
        to_phys(b, phi_);
        int mask = 0;
        for (int k = 0; k < dims; ++k) mask |= 1 << t[k];
        return ls_box(L, plo, phi_, mask);
    };
    auto coarse_box = [&](long long cb, double* rlo, double* rhi) {
        const int ci[3] = {(int)(cb % S1), (int)((cb / S1) % S1), (int)(cb / ((long long)S1 * S1))};
        for (int k = 0; k < dims; ++k) {
            rlo[k] = -1.0 + 2.0 * ci[k] / S1;
            rhi[k] = rlo[k] + 2.0 / S1;
        }
    };
    // 3-point Gauss rule per direction on the box; on a cut box, the species indicator at the node
    auto integrate = [&](const double* lo, const double* hi, bool cut) {
        const int nq = (dims == 3) ? 27 : 9;
        for (int q = 0; q < nq; ++q) {
            const int qi[3] = {q % 3, (q / 3) % 3, q / 9};
            double rr[3], wq = 1.0;
            for (int k = 0; k < dims; ++k) {
                const double hh = hi[k] - lo[k];
                rr[k] = lo[k] + 0.5 * hh * (sub.gx[qi[k]] + 1.0);
                wq *= 0.5 * hh * sub.gw[qi[k]];
            }
            if (cut) {
                double x[3];
                to_phys(rr, x);
                const double ph = ls_phi(L, x);
                if ((it.sp < 0) ? !(ph < 0.0) : (ph < 0.0)) continue;
            }
            double v[M];
            if (DIMS == 3) basis3(PD, rr, v);
            else basis2(PD, rr, v);
#pragma unroll
            for (int m = 0; m < M; ++m) acc[m] += wq * v[m];
        }
    };
    // Coarse boxes in chunks: (1) every thread classifies coarse boxes, integrates the uncut
    // ones of the species and lists the cut ones; (2) the (cut coarse box, fine box) pairs are
    // spread evenly over the block's threads, so the refinement work is balanced.
    constexpr int CHUNK = 1024;
    for (long long base = 0; base < ncoarse; base += CHUNK) {
        const int nb = (int)((ncoarse - base) < CHUNK ? (ncoarse - base) : CHUNK);
        if (threadIdx.x == 0) ncut = 0;
        __syncthreads();
        for (int i = threadIdx.x; i < nb; i += blockDim.x) {
            double rlo[3], rhi[3];
            coarse_box(base + i, rlo, rhi);
            const int cls = classify(rlo, rhi);
            if (cls == -it.sp) continue;   // fully in the other species
            if (cls == 0) {
                cutlist[atomicAdd(&ncut, 1)] = i;
                continue;
            }
            integrate(rlo, rhi, false);
        }
        __syncthreads();
        const long long work = (long long)ncut * nfine;
        for (long long wi = threadIdx.x; wi < work; wi += blockDim.x) {
            double rlo[3], rhi[3], flo[3], fhi[3];
            coarse_box(base + cutlist[wi / nfine], rlo, rhi);
            const long long fb = wi % nfine;
            const int fi[3] = {(int)(fb % S2), (int)((fb / S2) % S2), (int)(fb / ((long long)S2 * S2))};
            for (int k = 0; k < dims; ++k) {
                const double hh = (rhi[k] - rlo[k]) / S2;
                flo[k] = rlo[k] + fi[k] * hh;
                fhi[k] = flo[k] + hh;
            }
            const int fcls = classify(flo, fhi);
            if (fcls == -it.sp) continue;
            integrate(flo, fhi, fcls == 0);
        }
        __syncthreads();
    }
    // block reduction
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int m = 0; m < M; ++m) {
        double v = acc[m];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[m][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < M) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[threadIdx.x][w];
        mom[(long long)r * XDG_MAXM + threadIdx.x] = s;
    }
}

// moments of one item accumulated by one CTA; out[m], m < nmodes(dim, p)
__global__ void __launch_bounds__(256, 2) k_moments(const CutItem* __restrict__ items, int nitems, LevelSetDev L, Sub sub,
                                                 double* __restrict__ mom) {
    const int r = blockIdx.x;
    if (r >= nitems) return;
    const CutItem it = items[r];
    __shared__ int cutlist[1024];
    __shared__ int ncut;
    __shared__ double red[XDG_MAXM][33];
    switch (it.dim * 8 + it.p) {
#define BOSSS_MOM_CASE(DD, PP) \
    case DD * 8 + PP: moments_item<PP, DD>(it, r, L, sub, mom, cutlist, ncut, red); break;
        BOSSS_MOM_CASE(3, 0) BOSSS_MOM_CASE(3, 1) BOSSS_MOM_CASE(3, 2) BOSSS_MOM_CASE(3, 3) BOSSS_MOM_CASE(3, 4)
        BOSSS_MOM_CASE(2, 0) BOSSS_MOM_CASE(2, 1) BOSSS_MOM_CASE(2, 2) BOSSS_MOM_CASE(2, 3) BOSSS_MOM_CASE(2, 4)
#undef BOSSS_MOM_CASE
        default: break;
    }
}

// ------------------------------------------------------------------ device: weight solve
// Per rule: A[m][j] = phi_m(node_j); Householder QR of A^T = Q R (columns in degree order,
// so the leading columns are the lower-degree system); the minimum-norm solution of
// A w = b is w = Q [R^-T b; 0] -- what DGELSY returns for full row rank. The fitted degree
// is the highest one whose columns are numerically independent and whose solution
// reproduces its moments to 1e-11 relative.
__global__ void k_weight_solve(const CutItem* __restrict__ items, int nitems, const double* __restrict__ nodes,
                               const double* __restrict__ mom, double* __restrict__ weights, int* __restrict__ deg_out,
                               double* __restrict__ resid) {
    const int r = blockIdx.x;
    if (r >= nitems) return;
    const CutItem it = items[r];
    const int n = it.nnodes;
    const int dims = it.dim;
    __shared__ double At[XDG_MAXN][XDG_MAXM + 1];   // A^T, Householder vectors below the diagonal
    __shared__ double Rd[XDG_MAXM], vtv[XDG_MAXM], cn[XDG_MAXM];
    __shared__ double z[XDG_MAXM], t[XDG_MAXN], red[32];
    __shared__ int kmax;
    const int Mmax = (dims == 3) ? nmodes3(it.p) : nmodes2(it.p);
    const int M = Mmax < n ? Mmax : n;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        double v[XDG_MAXM];
        const double* xi = nodes + (it.node_off + j) * 3;
        if (dims == 3) basis3(it.p, xi, v);
        else basis2(it.p, xi, v);
        for (int m = 0; m < Mmax; ++m) At[j][m] = v[m];
    }
    __syncthreads();
    if (threadIdx.x < M) {
        double s = 0.0;
        for (int j = 0; j < n; ++j) s += At[j][threadIdx.x] * At[j][threadIdx.x];
        cn[threadIdx.x] = sqrt(s);
    }
    if (threadIdx.x == 0) kmax = M;
    __syncthreads();
    double cmax = 0.0;
    for (int m = 0; m < M; ++m) cmax = fmax(cmax, cn[m]);
    for (int k = 0; k < M; ++k) {
        if (threadIdx.x == 0) {
            double s = 0.0;
            for (int i = k; i < n; ++i) s += At[i][k] * At[i][k];
            const double nx = sqrt(s);
            if (!(nx > 1e-11 * cmax)) {
                kmax = k;
            } else {
                const double alpha = (At[k][k] >= 0.0) ? -nx : nx;
                At[k][k] -= alpha;
                vtv[k] = s - 2.0 * alpha * (At[k][k] + alpha) + alpha * alpha;   // |x - alpha e1|^2
                Rd[k] = alpha;
            }
        }
        __syncthreads();
        if (kmax <= k) break;
        for (int j = k + 1 + threadIdx.x; j < M; j += blockDim.x) {
            double s = 0.0;
            for (int i = k; i < n; ++i) s += At[i][k] * At[i][j];
            const double f = 2.0 * s / vtv[k];
            for (int i = k; i < n; ++i) At[i][j] -= f * At[i][k];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double* b = mom + (long long)r * XDG_MAXM;
        double bmax = 0.0;
        for (int m = 0; m < Mmax; ++m) bmax = fmax(bmax, fabs(b[m]));
        // highest degree with all its columns independent
        int pe = -1;
        for (int p = 0; p <= it.p; ++p)
            if (((dims == 3) ? nmodes3(p) : nmodes2(p)) <= kmax) pe = p;
        double res = 0.0;
        for (; pe >= 0; --pe) {
            const int me = (dims == 3) ? nmodes3(pe) : nmodes2(pe);
            // R^T z = b  (R[l][k] = At[l][k] for l < k, R[k][k] = Rd[k])
            for (int k = 0; k < me; ++k) {
                double s = b[k];
                for (int l = 0; l < k; ++l) s -= At[l][k] * z[l];
                z[k] = s / Rd[k];
            }
            for (int i = 0; i < n; ++i) t[i] = (i < me) ? z[i] : 0.0;
            for (int k = me - 1; k >= 0; --k) {   // t = H_0 ... H_{me-1} [z; 0]
                double s = 0.0;
                for (int i = k; i < n; ++i) s += At[i][k] * t[i];
                const double f = 2.0 * s / vtv[k];
                for (int i = k; i < n; ++i) t[i] -= f * At[i][k];
            }
            // residual of the fitted moments with the original basis values
            res = 0.0;
            const double* xb = nodes + it.node_off * 3;
            for (int m = 0; m < me; ++m) red[m & 31] = 0.0;
            double acc[XDG_MAXM];
            for (int m = 0; m < me; ++m) acc[m] = 0.0;
            for (int j = 0; j < n; ++j) {
                double v[XDG_MAXM];
                if (dims == 3) basis3(it.p, xb + j * 3, v);
                else basis2(it.p, xb + j * 3, v);
                for (int m = 0; m < me; ++m) acc[m] += v[m] * t[j];
            }
            for (int m = 0; m < me; ++m) res = fmax(res, fabs(acc[m] - b[m]));
            if (res <= 1e-11 * fmax(bmax, 1e-300)) break;
        }
        if (pe < 0) {   // degree 0 from the first column only
            pe = 0;
            double s = 0.0, v0 = 0.0;
            const double* xb = nodes + it.node_off * 3;
            for (int j = 0; j < n; ++j) {
                double v[XDG_MAXM];
                if (dims == 3) basis3(it.p, xb + j * 3, v);
                else basis2(it.p, xb + j * 3, v);
                s += v[0] * v[0];
                t[j] = v[0];
            }
            v0 = b[0] / s;
            for (int j = 0; j < n; ++j) t[j] *= v0;
            res = 0.0;
        }
        deg_out[r] = pe;
        resid[r] = res / fmax(bmax, 1e-300);
    }
    __syncthreads();
    for (int j = threadIdx.x; j < n; j += blockDim.x) weights[it.node_off + j] = t[j];
}

// ------------------------------------------------------------------ device: cut-rule evaluation
// Residual contributions of the cut items of one species, added with atomics:
// volume items: int_{K cap s} (fV v + fG . grad v) with the item's rule;
// face items: the SIP edge form on the cut face part (both cells, or boundary).
// Exponents (a, b, c) of basis function n in the reference order (degree-major, then a, then b):
// phi_n = L_a(x) L_b(y) L_c(z). With n a compile-time constant (unrolled loops) this folds away,
// so the per-node basis values and gradients live in registers instead of per-thread arrays.
template <int K>
__device__ __forceinline__ void mode3(int n, int& a, int& b, int& c) {
    int m = 0;
    a = b = c = 0;
#pragma unroll
    for (int deg = 0; deg <= K; ++deg)
#pragma unroll
        for (int aa = 0; aa <= deg; ++aa)
#pragma unroll
            for (int bb = 0; bb <= deg - aa; ++bb) {
                if (m == n) {
                    a = aa;
                    b = bb;
                    c = deg - aa - bb;
                }
                ++m;
            }
}

template <int K>
__device__ __forceinline__ double bphi(const double (&L)[3][K + 1], int n) {
    int a, b, c;
    mode3<K>(n, a, b, c);
    return L[0][a] * L[1][b] * L[2][c];
}

template <int K>
__device__ __forceinline__ double bgrad(const double (&L)[3][K + 1], const double (&dL)[3][K + 1], int n, int d) {
    int a, b, c;
    mode3<K>(n, a, b, c);
    if (d == 0) return dL[0][a] * L[1][b] * L[2][c];
    if (d == 1) return L[0][a] * dL[1][b] * L[2][c];
    return L[0][a] * L[1][b] * dL[2][c];
}

template <int K>
__global__ void k_cut_eval(const CutItem* __restrict__ items, int nitems, const double* __restrict__ nodes,
                           const double* __restrict__ weights, EvalArgs a, double* __restrict__ item_out) {
    using Phys = PhysScalar<3, true>;
    constexpr int NP = np_of(3, K);
    const int r = blockIdx.x;
    if (r >= nitems) return;
    const CutItem it = items[r];
    const GridConst& g = a.g;
    __shared__ double cA[NP], cB[NP];
    int ijk[3];
    cell_ijk(g, it.cell, ijk);
    long long other = -1;
    if (it.dim == 2) other = neighbour(g, ijk, it.dir, it.side);
    for (int n = threadIdx.x; n < NP; n += blockDim.x) {
        cA[n] = a.U[it.cell * NP + n];
        cB[n] = (other >= 0) ? a.U[other * NP + n] : 0.0;
    }
    __syncthreads();
    double rA[NP], rB[NP];
    for (int n = 0; n < NP; ++n) rA[n] = rB[n] = 0.0;
    const double sc = g.scaling;
    for (int j = threadIdx.x; j < it.nnodes; j += blockDim.x) {
        const double* t = nodes + (it.node_off + j) * 3;
        const double wq = weights[it.node_off + j];
        // reference coordinates of the node in the own cell (and the neighbour)
        double xiA[3], xiB[3];
        if (it.dim == 3) {
            xiA[0] = t[0];
            xiA[1] = t[1];
            xiA[2] = t[2];
        } else {
            const int t1 = (it.dir == 0) ? 1 : 0, t2 = (it.dir == 2) ? 1 : 2;
            xiA[it.dir] = it.side ? 1.0 : -1.0;
            xiA[t1] = t[0];
            xiA[t2] = t[1];
            xiB[it.dir] = -xiA[it.dir];
            xiB[t1] = t[0];
            xiB[t2] = t[1];
        }
        double LA[3][K + 1], dLA[3][K + 1], LB[3][K + 1], dLB[3][K + 1];
        for (int d = 0; d < 3; ++d) {
            legendre_vals(K, xiA[d], LA[d], dLA[d]);
            if (it.dim == 2) legendre_vals(K, xiB[d], LB[d], dLB[d]);
        }
        double uA = 0.0, GA[1][3] = {{0.0, 0.0, 0.0}};
#pragma unroll
        #pragma unroll
        for (int n = 0; n < NP; ++n) {
            uA += cA[n] * bphi<K>(LA, n);
            for (int d = 0; d < 3; ++d) GA[0][d] += cA[n] * bgrad<K>(LA, dLA, n, d);
        }
        uA *= sc;
        for (int d = 0; d < 3; ++d) GA[0][d] *= sc * g.twoh[d];
        double x[3];
        for (int d = 0; d < 3; ++d) x[d] = g.lo[d] + (ijk[d] + 0.5 + 0.5 * xiA[d]) * g.h[d];
        if (it.dim == 3) {
            double U1[1] = {uA}, fV[1] = {0.0}, fG[1][3] = {{0.0, 0.0, 0.0}};
            Phys::volume(a.ph, U1, GA, x, fV, fG);
            const double fac = wq * g.detJ * sc;
            #pragma unroll
            for (int n = 0; n < NP; ++n) {
                double acc = fV[0] * bphi<K>(LA, n);
                for (int d = 0; d < 3; ++d) acc += fG[0][d] * bgrad<K>(LA, dLA, n, d) * g.twoh[d];
                rA[n] += fac * acc;
            }
        } else {
            const double fac = wq * g.faceSG[it.dir] * sc;
            double nrm[3] = {0.0, 0.0, 0.0};
            if (other >= 0) {
                double uB = 0.0, GB[1][3] = {{0.0, 0.0, 0.0}};
                #pragma unroll
                for (int n = 0; n < NP; ++n) {
                    uB += cB[n] * bphi<K>(LB, n);
                    for (int d = 0; d < 3; ++d) GB[0][d] += cB[n] * bgrad<K>(LB, dLB, n, d);
                }
                uB *= sc;
                for (int d = 0; d < 3; ++d) GB[0][d] *= sc * g.twoh[d];
                // reference roles: IN = lower cell, normal +e_dir
                const bool selfLower = it.side == 1;
                nrm[it.dir] = 1.0;
                int ijk2[3] = {ijk[0], ijk[1], ijk[2]};
                ijk2[it.dir] = (int)((other / g.stride[it.dir]) % g.n[it.dir]);
                const double pnlty = a.ph.pen * fmax(penalty_size(a.cell_pf, g, ijk), penalty_size(a.cell_pf, g, ijk2));
                double U_in[1], U_out[1], G_in[1][3], G_out[1][3];
                U_in[0] = selfLower ? uA : uB;
                U_out[0] = selfLower ? uB : uA;
                for (int d = 0; d < 3; ++d) {
                    G_in[0][d] = selfLower ? GA[0][d] : GB[0][d];
                    G_out[0][d] = selfLower ? GB[0][d] : GA[0][d];
                }
                double gi[1] = {0.0}, go[1] = {0.0}, Gi[1][3] = {{0, 0, 0}}, Go[1][3] = {{0, 0, 0}};
                Phys::inner(a.ph, pnlty, U_in, G_in, U_out, G_out, nrm, x, gi, Gi, go, Go);
                // own cell A gets IN terms if it is the lower cell
                const double gsA = selfLower ? gi[0] : go[0], gsB = selfLower ? go[0] : gi[0];
                const double* GsA = selfLower ? Gi[0] : Go[0];
                const double* GsB = selfLower ? Go[0] : Gi[0];
                #pragma unroll
                for (int n = 0; n < NP; ++n) {
                    double accA = gsA * bphi<K>(LA, n), accB = gsB * bphi<K>(LB, n);
                    for (int d = 0; d < 3; ++d) {
                        accA += GsA[d] * bgrad<K>(LA, dLA, n, d) * g.twoh[d];
                        accB += GsB[d] * bgrad<K>(LB, dLB, n, d) * g.twoh[d];
                    }
                    rA[n] += fac * accA;
                    rB[n] += fac * accB;
                }
            } else {
                nrm[it.dir] = it.side ? 1.0 : -1.0;
                const double pnlty = 2.0 * a.ph.pen * penalty_size(a.cell_pf, g, ijk);
                double U1[1] = {uA}, gi[1] = {0.0}, Gi[1][3] = {{0, 0, 0}};
                Phys::boundary(a.ph, pnlty, U1, GA, nrm, x, nullptr, 0, gi, Gi);
                #pragma unroll
                for (int n = 0; n < NP; ++n) {
                    double acc = gi[0] * bphi<K>(LA, n);
                    for (int d = 0; d < 3; ++d) acc += Gi[0][d] * bgrad<K>(LA, dLA, n, d) * g.twoh[d];
                    rA[n] += fac * acc;
                }
            }
        }
    }
    // fixed-order reduction over the block (2 warps): warp shuffles, then the two warps' sums;
    // the item's contributions go to its slot of item_out (own cell, then the face
    // neighbour), which k_cut_gather adds into the cells in a fixed order -- no atomics, so
    // the result is the same bits run to run
    __shared__ double red[2][2][NP];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    #pragma unroll
    for (int n = 0; n < NP; ++n) {
        double va = rA[n], vb = rB[n];
        for (int o = 16; o > 0; o >>= 1) {
            va += __shfl_down_sync(0xffffffffu, va, o);
            vb += __shfl_down_sync(0xffffffffu, vb, o);
        }
        if (lane == 0) {
            red[warp][0][n] = va;
            red[warp][1][n] = vb;
        }
    }
    __syncthreads();
    const bool two = it.dim == 2 && other >= 0;
    for (int n = threadIdx.x; n < NP; n += blockDim.x) {
        item_out[((long long)r * 2 + 0) * NP + n] = a.alpha * (red[0][0][n] + red[1][0][n]);
        item_out[((long long)r * 2 + 1) * NP + n] = two ? a.alpha * (red[0][1][n] + red[1][1][n]) : 0.0;
    }
}

// out[cell] += the cut items' contributions to the cell, in item order (cells of the gather
// list: g_cell[i], sources g_src[g_off[i] .. g_off[i+1]) = item * 2 + side)
template <int K>
__global__ void k_cut_gather(long long ncells, const long long* __restrict__ g_off, const long long* __restrict__ g_cell,
                             const long long* __restrict__ g_src, const double* __restrict__ item_out,
                             double* __restrict__ out) {
    constexpr int NP = np_of(3, K);
    const long long n = ncells * NP;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const long long i = t / NP;
        const int m = (int)(t - i * NP);
        double acc = 0.0;
        for (long long e = g_off[i]; e < g_off[i + 1]; ++e) acc += item_out[g_src[e] * NP + m];
        out[g_cell[i] * NP + m] += acc;
    }
}

// ------------------------------------------------------------------ level-set interface term
// XLaplace_Interface.InnerEdgeForm (XNSECommon/XLaplace.cs:229-297) integrated over the sphere
// surface inside each cut cell, scattered into both species' rows of the cell as
// NECQuadratureLevelSet.SaveIntegrationResults does (NECQuadratureLevelSet.cs:622-661): the form
// with (vA, vB) = (phi_n, 0) goes to species A, with (0, phi_n) to species B, both added. The
// normal is the level-set normal grad(phi)/|grad(phi)|, pointing from A (phi < 0) to B.
// One block per cut cell; every cell occurs once, so the block adds its sums without atomics.
struct IfaceArgs {
    double muA, muB;     // species diffusivities
    double omA, omB;     // flux weights (SIP 1/2, 1/2; SWIP muB/(muA+muB), muA/(muA+muB))
    double pen;          // penalty_base * penalty_deg * penalty_muFactor (times the size factor per cell)
    double alpha;
    // the species' penalty size factors (1 / cell length scale, per cell): the interface penalty
    // takes max(pfA[j], pfB[j]) of the cut cell (XLaplace_Interface.GetPenalty, XLaplace.cs:261-297)
    const double* pfA;
    const double* pfB;
};

template <int K>
__global__ void k_interface_eval(const long long* __restrict__ cells, const long long* __restrict__ node_off,
                                 const double* __restrict__ nodes, const double* __restrict__ weights,
                                 const double* __restrict__ normals, int ncells, GridConst g, IfaceArgs f,
                                 const double* __restrict__ UA, const double* __restrict__ UB, double* outA,
                                 double* outB) {
    constexpr int NP = np_of(3, K);
    const int r = blockIdx.x;
    if (r >= ncells) return;
    const long long cell = cells[r];
    __shared__ double cA[NP], cB[NP], RA[NP], RB[NP];
    for (int n = threadIdx.x; n < NP; n += blockDim.x) {
        cA[n] = UA[cell * NP + n];
        cB[n] = UB[cell * NP + n];
        RA[n] = 0.0;
        RB[n] = 0.0;
    }
    __syncthreads();
    const double pen = f.pen * fmax(f.pfA[cell], f.pfB[cell]);
    const double sc = g.scaling;
    double rA[NP], rB[NP];
    for (int n = 0; n < NP; ++n) rA[n] = rB[n] = 0.0;
    const long long j0 = node_off[r], j1 = node_off[r + 1];
    for (long long j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
        const double* xi = nodes + 3 * j;
        const double* N = normals + 3 * j;
        double L[3][K + 1], dL[3][K + 1];
        for (int d = 0; d < 3; ++d) legendre_vals(K, xi[d], L[d], dL[d]);
        double ph[NP], gn[NP];   // basis value and normal derivative (physical, without sc)
        double uA = 0.0, uB = 0.0, gA = 0.0, gB = 0.0;
        {
            int nn = 0;
            for (int deg = 0; deg <= K; ++deg)
                for (int aa = 0; aa <= deg; ++aa)
                    for (int bb = 0; bb <= deg - aa; ++bb) {
                        const int cc = deg - aa - bb;
                        ph[nn] = L[0][aa] * L[1][bb] * L[2][cc];
                        gn[nn] = dL[0][aa] * L[1][bb] * L[2][cc] * g.twoh[0] * N[0] +
                                 L[0][aa] * dL[1][bb] * L[2][cc] * g.twoh[1] * N[1] +
                                 L[0][aa] * L[1][bb] * dL[2][cc] * g.twoh[2] * N[2];
                        uA += cA[nn] * ph[nn];
                        uB += cB[nn] * ph[nn];
                        gA += cA[nn] * gn[nn];
                        gB += cB[nn] * gn[nn];
                        ++nn;
                    }
        }
        uA *= sc;
        uB *= sc;
        gA *= sc;
        gB *= sc;
        const double jump = uA - uB;
        const double flux = f.muA * f.omA * gA + f.muB * f.omB * gB - pen * jump;
        const double w = weights[j] * sc;
        const double symA = f.muA * f.omA * jump, symB = f.muB * f.omB * jump;
        for (int n = 0; n < NP; ++n) {
            rA[n] += w * (flux * ph[n] + symA * gn[n]);
            rB[n] += w * (-flux * ph[n] + symB * gn[n]);
        }
    }
    // fixed-order reduction over the block (2 warps of 32): the same bits run to run
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int n = 0; n < NP; ++n) {
        double va = rA[n], vb = rB[n];
        for (int o = 16; o > 0; o >>= 1) {
            va += __shfl_down_sync(0xffffffffu, va, o);
            vb += __shfl_down_sync(0xffffffffu, vb, o);
        }
        if (lane == 0 && warp == 1) {
            RA[n] = va;
            RB[n] = vb;
        }
        if (lane == 0 && warp == 0) {
            rA[n] = va;
            rB[n] = vb;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int n = 0; n < NP; ++n) {
            outA[cell * NP + n] += f.alpha * (rA[n] + RA[n]);
            outB[cell * NP + n] += f.alpha * (rB[n] + RB[n]);
        }
}

// Surface rule of the sphere |x - c| = R inside the box [lo, hi] (physical coordinates), by
// height-function quadrature with analytic roots (the approach of Saye's high-order rules,
// Quadrature/SayeGaussRule_*.cs, specialised to the quadric): a height direction m with c_m
// outside [lo_m, hi_m] makes the surface one graph x_m = c_m + s sqrt(R^2 - rho^2) over the base
// plane (a, b); the inner integral over b runs over the intervals where the root lies in the box,
// the outer integral over a is split where those intervals change shape, and each outer piece is
// mapped by a = a0 + (a1 - a0)(3u^2 - 2u^3) so that square-root behaviour at its ends becomes
// smooth. dS = R / |x_m - c_m| dA. Boxes with no admissible height direction are halved in every
// direction. Appends (x[3], w, n[3]) per node.
static void sphere_surface_box(const double* lo, const double* hi, const double* c, double R,
                               const std::vector<double>& gx, const std::vector<double>& gw, int depth,
                               std::vector<double>& out) {
    LevelSetDev L{};
    L.type = BOSSS_LEVELSET_SPHERE;
    for (int d = 0; d < 3; ++d) L.c[d] = c[d];
    L.r = R;
    if (ls_box(L, lo, hi, 7) != 0) return;
    int m = -1;
    double best = 0.0;
    for (int d = 0; d < 3; ++d) {
        const double dist = std::max(lo[d] - c[d], c[d] - hi[d]);
        if (dist > best) {
            best = dist;
            m = d;
        }
    }
    if (m < 0) {
        if (depth >= 6) return;
        double mid[3];
        for (int d = 0; d < 3; ++d) mid[d] = 0.5 * (lo[d] + hi[d]);
        for (int q = 0; q < 8; ++q) {
            double l2[3], h2[3];
            for (int d = 0; d < 3; ++d) {
                const bool up = (q >> d) & 1;
                l2[d] = up ? mid[d] : lo[d];
                h2[d] = up ? hi[d] : mid[d];
            }
            sphere_surface_box(l2, h2, c, R, gx, gw, depth + 1, out);
        }
        return;
    }
    const int a = (m == 0) ? 1 : 0, b = (m == 2) ? 1 : 2;
    const double s = (lo[m] > c[m]) ? 1.0 : -1.0;
    const double dlo = best;
    const double dhi = std::max(std::fabs(lo[m] - c[m]), std::fabs(hi[m] - c[m]));
    // break points of the outer direction
    std::vector<double> br = {lo[a], hi[a]};
    const double ds[2] = {dlo, dhi};
    const double es[3] = {lo[b] - c[b], hi[b] - c[b], 0.0};
    for (double dd : ds)
        for (double ee : es) {
            const double q = R * R - dd * dd - ee * ee;
            if (q <= 0.0) continue;
            const double t = std::sqrt(q);
            for (double xa : {c[a] - t, c[a] + t})
                if (xa > lo[a] && xa < hi[a]) br.push_back(xa);
        }
    std::sort(br.begin(), br.end());
    const int n = (int)gx.size();
    for (size_t ia = 0; ia + 1 < br.size(); ++ia) {
        const double a0 = br[ia], a1 = br[ia + 1];
        if (!(a1 > a0)) continue;
        for (int i = 0; i < n; ++i) {
            const double u = 0.5 * (gx[i] + 1.0);
            const double xa = a0 + (a1 - a0) * u * u * (3.0 - 2.0 * u);
            const double wa = 0.5 * gw[i] * (a1 - a0) * 6.0 * u * (1.0 - u);
            const double A = R * R - (xa - c[a]) * (xa - c[a]);
            const double ro2 = A - dlo * dlo;
            if (ro2 <= 0.0) continue;
            const double ro = std::sqrt(ro2), ri = std::sqrt(std::max(0.0, A - dhi * dhi));
            const double iv[2][2] = {{c[b] - ro, c[b] - ri}, {c[b] + ri, c[b] + ro}};
            for (int k = 0; k < 2; ++k) {
                const double b0 = std::max(iv[k][0], lo[b]), b1 = std::min(iv[k][1], hi[b]);
                if (!(b1 > b0)) continue;
                for (int jn = 0; jn < n; ++jn) {
                    const double xb = 0.5 * (b0 + b1) + 0.5 * (b1 - b0) * gx[jn];
                    const double wb = 0.5 * (b1 - b0) * gw[jn];
                    const double D = A - (xb - c[b]) * (xb - c[b]);
                    const double hgt = std::sqrt(std::max(D, dlo * dlo));
                    double x[3];
                    x[a] = xa;
                    x[b] = xb;
                    x[m] = c[m] + s * std::min(std::max(hgt, dlo), dhi);
                    const double rr = std::sqrt((x[0] - c[0]) * (x[0] - c[0]) + (x[1] - c[1]) * (x[1] - c[1]) +
                                                (x[2] - c[2]) * (x[2] - c[2]));
                    const double w = wa * wb * R / std::fabs(x[m] - c[m]);
                    out.push_back(x[0]);
                    out.push_back(x[1]);
                    out.push_back(x[2]);
                    out.push_back(w);
                    for (int d = 0; d < 3; ++d) out.push_back((x[d] - c[d]) / rr);
                }
            }
        }
    }
}

}  // namespace bosss

namespace bosss {
// out[i] *= beta on [0, n): the cells outside a species' band take no contribution
__global__ void k_scale(double* __restrict__ out, long long n, double beta) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] *= beta;
}
}  // namespace bosss

using namespace bosss;

struct bosss_xdg {
    int device = 0;
    bosss_handle* h[2] = {nullptr, nullptr};   // species A (phi < 0), B (phi > 0)
    LevelSetDev ls{};
    int K = 0;
    // per species: masks and cut items
    unsigned char* d_vol[2] = {nullptr, nullptr};
    unsigned char* d_face[2] = {nullptr, nullptr};
    std::vector<unsigned char> vol[2], face[2];
    std::vector<CutItem> items[2];
    CutItem* d_items[2] = {nullptr, nullptr};
    // deterministic accumulation of the cut items: per-item outputs (item, side, NP) and the
    // per-cell gather lists (cells, CSR offsets, sources item * 2 + side, in item order)
    double* d_item_out[2] = {nullptr, nullptr};
    long long* d_g_off[2] = {nullptr, nullptr};
    long long* d_g_cell[2] = {nullptr, nullptr};
    long long* d_g_src[2] = {nullptr, nullptr};
    long long n_gcells[2] = {0, 0};
    double* d_nodes[2] = {nullptr, nullptr};
    double* d_weights[2] = {nullptr, nullptr};
    std::vector<double> nodes[2], weights[2];
    std::vector<int> fitted_deg[2];
    std::vector<double> fit_resid[2];
    std::vector<double> moments[2];   // XDG_MAXM per item
    long long n_cells[2] = {0, 0};
    // per species: the cells [rng[s][0], rng[s][1]) hold every cell with species content (cells
    // are in generator order, so a species inside a sphere spans a band of x-planes)
    long long rng[2][2] = {{0, 0}, {0, 0}};
    // species B on the unmasked slab kernel outside [sb[0], sb[1]): whole x-planes whose cells
    // are all uncut species-B cells with standard faces (null: the slab kernel is not available)
    bosss_handle* hs = nullptr;
    long long sb[2] = {0, 0};
    // per species: cell length scales of the SIP penalty (computed defaults, and the ones in
    // use: the defaults or the caller's), penalty size factors 1/len on the device
    std::vector<double> len_default[2], len[2];
    double* d_pf[2] = {nullptr, nullptr};
    // level-set interface term (set by bosss_b200_xdg_interface_setup)
    bool iface = false;
    IfaceArgs ifa{};
    std::vector<long long> if_cells, if_off;
    std::vector<double> if_nodes, if_w, if_n;   // reference coordinates, weights, normals
    long long* d_if_cells = nullptr;
    long long* d_if_off = nullptr;
    double* d_if_nodes = nullptr;
    double* d_if_w = nullptr;
    double* d_if_n = nullptr;
};

namespace bosss {

// ---------------------------------------------------------------------------------------
// Saye-type rules for the species part of a cut cell or cut face (the reference's default
// rule family, SayeGaussRule_Algorithm.cs / _Cube.cs / _Square.cs, after R. Saye, "High-order
// quadrature methods for implicitly defined surfaces and volumes in hyperrectangles", SIAM J.
// Sci. Comput. 37 (2015)), written for the sphere level set in reference coordinates of the
// item ([-1,1]^dim). Recursion over the free directions of a box: functions with one sign on
// the box are dropped (or empty the box, if the sign is the wrong one); with none left, a
// tensor Gauss rule; else a height direction k in which every function is strictly monotone
// (the largest |d phi / d x_k| at the centre among those), the functions restricted to the two
// faces x_k = lo_k, hi_k become the (sign-free, split-only) functions of the box without k,
// whose rule is built recursively; at each of its nodes the line in direction k is split at
// the functions' roots and the pieces with the required sign get a Gauss rule. Boxes without
// such a direction are halved in every free direction (at most 8 times; then a tensor rule
// filtered by the sign at the nodes).
struct SayeFn {
    unsigned fixmask;   // reference directions fixed at fixval
    double fixval[3];
    int sign;           // required sign of phi (+1 / -1), 0: split only
};

struct SayeItem {
    const LevelSetDev* L;
    int dim, dir, sp;
    double center[3], h[3];
    const std::vector<double>* gx;
    const std::vector<double>* gw;
    std::vector<double>* nodes;   // 3 per node (reference coordinates)
    std::vector<double>* weights;
    // physical point of the full reference coordinates r (dim entries used)
    void phys(const double* r, double* x) const {
        for (int d = 0; d < 3; ++d) x[d] = center[d];
        if (dim == 3) {
            for (int d = 0; d < 3; ++d) x[d] += 0.5 * h[d] * r[d];
        } else {
            const int t1 = (dir == 0) ? 1 : 0, t2 = (dir == 2) ? 1 : 2;
            x[t1] += 0.5 * h[t1] * r[0];
            x[t2] += 0.5 * h[t2] * r[1];
        }
    }
    int pdir(int k) const {   // physical direction of reference direction k
        if (dim == 3) return k;
        const int t1 = (dir == 0) ? 1 : 0, t2 = (dir == 2) ? 1 : 2;
        return k == 0 ? t1 : t2;
    }
    double value(const SayeFn& f, const double* r) const {
        double rr[3] = {r[0], r[1], r[2]}, x[3];
        for (int d = 0; d < dim; ++d)
            if (f.fixmask & (1u << d)) rr[d] = f.fixval[d];
        phys(rr, x);
        return ls_phi(*L, x);
    }
    // physical box of f over the reference box [lo, hi] (fixed directions degenerate)
    void pbox(const SayeFn& f, const double* lo, const double* hi, double* plo, double* phi_, int& mask) const {
        double a[3] = {lo[0], lo[1], lo[2]}, b[3] = {hi[0], hi[1], hi[2]};
        for (int d = 0; d < dim; ++d)
            if (f.fixmask & (1u << d)) a[d] = b[d] = f.fixval[d];
        double xa[3], xb[3];
        phys(a, xa);
        phys(b, xb);
        mask = 0;
        for (int d = 0; d < 3; ++d) {
            plo[d] = std::min(xa[d], xb[d]);
            phi_[d] = std::max(xa[d], xb[d]);
            if (phi_[d] > plo[d]) mask |= 1 << d;
        }
    }
    int sign_on(const SayeFn& f, const double* lo, const double* hi) const {
        double plo[3], phi_[3];
        int mask;
        pbox(f, lo, hi, plo, phi_, mask);
        return ls_box(*L, plo, phi_, mask);
    }
    // usable height direction k over the box: the sphere's d phi / d x_m = (x_m - c_m) / |x - c|
    // keeps its sign iff c_m lies outside the physical range; it is also kept away from zero by
    // asking c_m to be at least a quarter of the box width outside (closer boxes are split, so
    // that the height function has no near-vertical tangent inside a piece)
    bool monotone(const SayeFn& f, const double* lo, const double* hi, int k) const {
        double plo[3], phi_[3];
        int mask;
        pbox(f, lo, hi, plo, phi_, mask);
        const int m = pdir(k);
        const double w = 0.25 * (phi_[m] - plo[m]);
        return L->c[m] < plo[m] - w || L->c[m] > phi_[m] + w;
    }
    double slope(const SayeFn& f, const double* r, int k) const {
        double rr[3] = {r[0], r[1], r[2]}, x[3];
        for (int d = 0; d < dim; ++d)
            if (f.fixmask & (1u << d)) rr[d] = f.fixval[d];
        phys(rr, x);
        const double dist = std::sqrt((x[0] - L->c[0]) * (x[0] - L->c[0]) + (x[1] - L->c[1]) * (x[1] - L->c[1]) +
                                      (x[2] - L->c[2]) * (x[2] - L->c[2]));
        const int m = pdir(k);
        return dist > 0.0 ? (x[m] - L->c[m]) / dist * 0.5 * h[m] : 0.0;
    }
};

// root of the monotone function t -> f(r with r[k] = t) in (a, b), f(a) f(b) < 0
static double saye_root(const SayeItem& S, const SayeFn& f, double* r, int k, double a, double b, double fa) {
    double lo = a, hi = b, flo = fa;
    for (int it = 0; it < 200 && hi - lo > 1e-15 * std::max(1.0, std::fabs(lo)); ++it) {
        const double m = 0.5 * (lo + hi);
        r[k] = m;
        const double fm = S.value(f, r);
        if (fm == 0.0) return m;
        if ((fm < 0.0) == (flo < 0.0)) {
            lo = m;
            flo = fm;
        } else {
            hi = m;
        }
    }
    return 0.5 * (lo + hi);
}

// emit(r, w): nodes of the free directions `free` (bit mask) of the box [lo, hi]; r holds
// the values of all directions, entries of non-free directions set by the caller
using SayeEmit = std::function<void(double*, double)>;
static void saye_box(const SayeItem& S, unsigned free, const double* lo, const double* hi, std::vector<SayeFn> fns,
                     int depth, double* r, const SayeEmit& emit);

static void saye_tensor(const SayeItem& S, unsigned free, const double* lo, const double* hi, double* r,
                        const std::vector<SayeFn>* filter, const SayeEmit& emit) {
    int dirs[3], nf = 0;
    for (int d = 0; d < S.dim; ++d)
        if (free & (1u << d)) dirs[nf++] = d;
    const std::vector<double>& gx = *S.gx;
    const std::vector<double>& gw = *S.gw;
    const int q = (int)gx.size();
    int tot = 1;
    for (int i = 0; i < nf; ++i) tot *= q;
    for (int t = 0; t < tot; ++t) {
        double w = 1.0;
        int u = t;
        for (int i = 0; i < nf; ++i) {
            const int d = dirs[i], j = u % q;
            u /= q;
            r[d] = 0.5 * (lo[d] + hi[d]) + 0.5 * (hi[d] - lo[d]) * gx[j];
            w *= 0.5 * (hi[d] - lo[d]) * gw[j];
        }
        bool ok = true;
        if (filter)
            for (const SayeFn& f : *filter)
                if (f.sign != 0) {
                    const double v = S.value(f, r);
                    if (f.sign < 0 ? !(v < 0.0) : (v < 0.0)) ok = false;
                }
        if (ok) emit(r, w);
    }
}

// 1D integration along k at the current r: split at the functions' roots, keep the pieces
// whose midpoint has every required sign
static void saye_line(const SayeItem& S, int k, double a, double b, const std::vector<SayeFn>& fns, double* r,
                      double w0, const SayeEmit& emit) {
    std::vector<double> br = {a, b};
    for (const SayeFn& f : fns) {
        r[k] = a;
        const double fa = S.value(f, r);
        r[k] = b;
        const double fb = S.value(f, r);
        if ((fa < 0.0) != (fb < 0.0) && fa != 0.0 && fb != 0.0) br.push_back(saye_root(S, f, r, k, a, b, fa));
    }
    std::sort(br.begin(), br.end());
    const std::vector<double>& gx = *S.gx;
    const std::vector<double>& gw = *S.gw;
    for (size_t i = 0; i + 1 < br.size(); ++i) {
        const double t0 = br[i], t1 = br[i + 1];
        if (!(t1 > t0)) continue;
        r[k] = 0.5 * (t0 + t1);
        bool ok = true;
        for (const SayeFn& f : fns)
            if (f.sign != 0) {
                const double v = S.value(f, r);
                if (f.sign < 0 ? !(v < 0.0) : (v < 0.0)) ok = false;
            }
        if (!ok) continue;
        for (size_t j = 0; j < gx.size(); ++j) {
            r[k] = 0.5 * (t0 + t1) + 0.5 * (t1 - t0) * gx[j];
            emit(r, w0 * 0.5 * (t1 - t0) * gw[j]);
        }
    }
}

static void saye_box(const SayeItem& S, unsigned free, const double* lo, const double* hi, std::vector<SayeFn> fns,
                     int depth, double* r, const SayeEmit& emit) {
    // drop functions of one sign on the box
    std::vector<SayeFn> live;
    for (const SayeFn& f : fns) {
        const int sg = S.sign_on(f, lo, hi);
        if (sg == 0) {
            live.push_back(f);
            continue;
        }
        if (f.sign != 0 && sg != f.sign) return;   // the box lies in the other species
    }
    if (live.empty()) {
        saye_tensor(S, free, lo, hi, r, nullptr, emit);
        return;
    }
    int nf = 0, only = -1;
    for (int d = 0; d < S.dim; ++d)
        if (free & (1u << d)) {
            ++nf;
            only = d;
        }
    if (nf == 1) {
        saye_line(S, only, lo[only], hi[only], live, r, 1.0, emit);
        return;
    }
    // height direction: every live function strictly monotone, largest slope of the first
    double rc[3] = {r[0], r[1], r[2]};
    for (int d = 0; d < S.dim; ++d)
        if (free & (1u << d)) rc[d] = 0.5 * (lo[d] + hi[d]);
    int k = -1;
    double best = -1.0;
    for (int d = 0; d < S.dim; ++d) {
        if (!(free & (1u << d))) continue;
        bool mono = true;
        for (const SayeFn& f : live) mono = mono && S.monotone(f, lo, hi, d);
        if (!mono) continue;
        const double sl = std::fabs(S.slope(live[0], rc, d));
        if (sl > best) {
            best = sl;
            k = d;
        }
    }
    if (k < 0) {
        if (depth >= 8) {
            saye_tensor(S, free, lo, hi, r, &live, emit);
            return;
        }
        const int nch = 1 << nf;
        for (int c = 0; c < nch; ++c) {
            double l2[3] = {lo[0], lo[1], lo[2]}, h2[3] = {hi[0], hi[1], hi[2]};
            int bit = 0;
            for (int d = 0; d < S.dim; ++d) {
                if (!(free & (1u << d))) continue;
                const double mid = 0.5 * (lo[d] + hi[d]);
                if ((c >> bit) & 1) l2[d] = mid;
                else h2[d] = mid;
                ++bit;
            }
            saye_box(S, free, l2, h2, live, depth + 1, r, emit);
        }
        return;
    }
    // reduced problem without k: the live functions on the two faces x_k = lo_k, hi_k
    std::vector<SayeFn> red;
    for (const SayeFn& f : live)
        for (int side = 0; side < 2; ++side) {
            SayeFn g = f;
            g.fixmask |= 1u << k;
            g.fixval[k] = side ? hi[k] : lo[k];
            g.sign = 0;
            red.push_back(g);
        }
    const double a = lo[k], b = hi[k];
    const SayeEmit inner = [&](double* rr, double w) { saye_line(S, k, a, b, live, rr, w, emit); };
    saye_box(S, free & ~(1u << k), lo, hi, red, depth, r, inner);
}

// Saye-type rule of an item's species part: appends nodes (reference coordinates, 3 per node)
// and weights (reference measure); returns the node count
static int saye_item_rule(const LevelSetDev& L, const CutItem& it, const std::vector<double>& gx,
                          const std::vector<double>& gw, std::vector<double>& nodes, std::vector<double>& weights) {
    SayeItem S;
    S.L = &L;
    S.dim = it.dim;
    S.dir = it.dir;
    S.sp = it.sp;
    for (int d = 0; d < 3; ++d) {
        S.center[d] = it.center[d];
        S.h[d] = it.h[d];
    }
    S.gx = &gx;
    S.gw = &gw;
    S.nodes = &nodes;
    S.weights = &weights;
    const double lo[3] = {-1.0, -1.0, it.dim == 3 ? -1.0 : 0.0}, hi[3] = {1.0, 1.0, it.dim == 3 ? 1.0 : 0.0};
    SayeFn f{};
    f.fixmask = 0;
    f.sign = it.sp;   // species A: phi < 0, B: phi >= 0
    const size_t n0 = weights.size();
    double r[3] = {0.0, 0.0, 0.0};
    const SayeEmit emit = [&](double* rr, double w) {
        nodes.push_back(rr[0]);
        nodes.push_back(rr[1]);
        nodes.push_back(it.dim == 3 ? rr[2] : 0.0);
        weights.push_back(w);
    };
    saye_box(S, it.dim == 3 ? 7u : 3u, lo, hi, {f}, 0, r, emit);
    return (int)(weights.size() - n0);
}

static int build_species(bosss_xdg* X, int s, const bosss_xdg_opts& xo) {
    const GridConst& g = X->h[s]->base.g;
    const int sp = s == 0 ? -1 : +1;
    const long long J = g.J;
    X->vol[s].assign(J, 0);
    X->face[s].assign(J * 6, 0);
    std::vector<double> gx5, gw5, gx9, gw9;
    gauss(xo.cut_nodes_1d, gx5, gw5);
    gauss(xo.fallback_nodes_1d, gx9, gw9);
    auto& items = X->items[s];
    auto& nodes = X->nodes[s];
    items.clear();
    nodes.clear();
    X->weights[s].clear();
    const int pmax = xo.moment_degree;
    auto add_item = [&](long long cell, int dim, int dir, int side, const double* center, const double* hh) {
        CutItem it{};
        it.cell = cell;
        it.dim = dim;
        it.dir = dir;
        it.side = side;
        it.sp = sp;
        it.p = pmax;
        for (int d = 0; d < 3; ++d) {
            it.center[d] = center[d];
            it.h[d] = hh[d];
        }
        if (xo.rule == 1) {   // Saye-type rule: nodes and weights directly
            it.node_off = (long long)nodes.size() / 3;
            it.nnodes = saye_item_rule(X->ls, it, gx5, gw5, nodes, X->weights[s]);
            items.push_back(it);
            return;
        }
        // candidate nodes: tensor Gauss nodes of the species part, finer set for small parts
        auto collect = [&](const std::vector<double>& gx, bool all) {
            std::vector<std::array<double, 3>> v;
            const int nq = (int)gx.size();
            const int tot = (dim == 3) ? nq * nq * nq : nq * nq;
            const int t1 = (dir == 0) ? 1 : 0, t2 = (dir == 2) ? 1 : 2;
            for (int q = 0; q < tot; ++q) {
                double rr[3] = {gx[q % nq], gx[(q / nq) % nq], (dim == 3) ? gx[q / (nq * nq)] : 0.0};
                double x[3];
                if (dim == 3) {
                    for (int d = 0; d < 3; ++d) x[d] = center[d] + 0.5 * hh[d] * rr[d];
                } else {
                    for (int d = 0; d < 3; ++d) x[d] = center[d];
                    x[t1] += 0.5 * hh[t1] * rr[0];
                    x[t2] += 0.5 * hh[t2] * rr[1];
                }
                const double ph = ls_phi(X->ls, x);
                if (all || ((sp < 0) ? (ph < 0.0) : !(ph < 0.0))) v.push_back({rr[0], rr[1], rr[2]});
            }
            return v;
        };
        // candidates: Gauss nodes inside the species part (5^D), a finer set (9^D) for small
        // parts, and for slivers without 8 such nodes the whole 5^D set (moment fitting does
        // not need the nodes inside the part: it integrates the polynomial extension)
        auto cand = collect(gx5, false);
        if ((int)cand.size() < 8) {
            auto c9 = collect(gx9, false);
            cand = ((int)c9.size() >= 8 && (int)c9.size() <= XDG_MAXN) ? c9 : collect(gx5, true);
        }
        if ((int)cand.size() > XDG_MAXN) cand.resize(XDG_MAXN);
        it.nnodes = (int)cand.size();
        it.node_off = (long long)nodes.size() / 3;
        for (auto& c : cand)
            for (int d = 0; d < 3; ++d) nodes.push_back(c[d]);
        items.push_back(it);
    };
    for (long long j = 0; j < J; ++j) {
        int ijk[3];
        for (int d = 0; d < 3; ++d) ijk[d] = (int)((j / g.stride[d]) % g.n[d]);
        double lo[3], hi[3], c[3];
        for (int d = 0; d < 3; ++d) {
            lo[d] = g.lo[d] + ijk[d] * g.h[d];
            hi[d] = lo[d] + g.h[d];
            c[d] = 0.5 * (lo[d] + hi[d]);
        }
        const int cls = ls_box(X->ls, lo, hi, 7);
        if (cls == sp) X->vol[s][j] = 1;
        else if (cls == 0) {
            X->vol[s][j] = 2;
            add_item(j, 3, 0, 0, c, g.h);
        }
        if (X->vol[s][j] == 0) continue;
        // faces of the cell
        for (int d = 0; d < 3; ++d)
            for (int side = 0; side < 2; ++side) {
                double flo[3], fhi[3], fc[3];
                for (int dd = 0; dd < 3; ++dd) {
                    flo[dd] = lo[dd];
                    fhi[dd] = hi[dd];
                    fc[dd] = c[dd];
                }
                flo[d] = fhi[d] = fc[d] = side ? hi[d] : lo[d];
                const int fcls = ls_box(X->ls, flo, fhi, 7 & ~(1 << d));
                unsigned char fl = 0;
                if (fcls == sp) fl = 1;
                else if (fcls == 0) fl = 2;
                X->face[s][j * 6 + 2 * d + side] = fl;
                if (fl == 2) {
                    // one item per cut face: interior faces from the lower cell, boundary faces from their cell
                    const bool boundary = !g.periodic[d] && ((side == 0 && ijk[d] == 0) || (side == 1 && ijk[d] == g.n[d] - 1));
                    if (boundary || side == 1) add_item(j, 2, d, side, fc, g.h);
                }
            }
    }
    long long cnt = 0;
    for (long long j = 0; j < J; ++j) cnt += X->vol[s][j] != 0;
    X->n_cells[s] = cnt;
    return BOSSS_OK;
}

static int upload_and_fit(bosss_xdg* X, int s, const bosss_xdg_opts& xo) {
    auto& items = X->items[s];
    const int n = (int)items.size();
    const size_t nn = X->nodes[s].size() / 3;
    CUDA_TRY(cudaMalloc(&X->d_vol[s], X->vol[s].size()));
    CUDA_TRY(cudaMalloc(&X->d_face[s], X->face[s].size()));
    CUDA_TRY(cudaMemcpy(X->d_vol[s], X->vol[s].data(), X->vol[s].size(), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(X->d_face[s], X->face[s].data(), X->face[s].size(), cudaMemcpyHostToDevice));
    const bool saye = xo.rule == 1;   // weights already set by the Saye-type rules
    if (!saye) X->weights[s].assign(nn, 0.0);
    X->fitted_deg[s].assign(n, -1);
    X->fit_resid[s].assign(n, 0.0);
    if (n == 0) return BOSSS_OK;
    CUDA_TRY(cudaMalloc(&X->d_items[s], sizeof(CutItem) * n));
    CUDA_TRY(cudaMalloc(&X->d_nodes[s], sizeof(double) * 3 * nn));
    CUDA_TRY(cudaMalloc(&X->d_weights[s], sizeof(double) * nn));
    CUDA_TRY(cudaMemcpy(X->d_items[s], items.data(), sizeof(CutItem) * n, cudaMemcpyHostToDevice));
    {
        // gather lists: every cell an item contributes to (its cell, and a cut face's neighbour)
        const GridConst& g = X->h[s]->base.g;
        std::vector<std::vector<long long>> src((size_t)g.J);
        std::vector<long long> touched;
        auto add = [&](long long cell, long long e) {
            if (src[cell].empty()) touched.push_back(cell);
            src[cell].push_back(e);
        };
        for (int r = 0; r < n; ++r) {
            const CutItem& it = items[r];
            add(it.cell, 2LL * r);
            if (it.dim != 2) continue;
            int ijk[3];
            for (int d = 0; d < 3; ++d) ijk[d] = (int)((it.cell / g.stride[d]) % g.n[d]);
            int i = ijk[it.dir] + (it.side ? 1 : -1);
            if (i < 0 || i >= g.n[it.dir]) {
                if (!g.periodic[it.dir]) continue;
                i = (i + g.n[it.dir]) % g.n[it.dir];
            }
            long long other = 0;
            for (int d = 0; d < 3; ++d) other += (long long)((d == it.dir) ? i : ijk[d]) * g.stride[d];
            add(other, 2LL * r + 1);
        }
        std::sort(touched.begin(), touched.end());
        std::vector<long long> off(1, 0), flat;
        for (long long c : touched) {
            flat.insert(flat.end(), src[c].begin(), src[c].end());
            off.push_back((long long)flat.size());
        }
        const int NP = np_of(3, X->K);
        X->n_gcells[s] = (long long)touched.size();
        CUDA_TRY(cudaMalloc(&X->d_item_out[s], sizeof(double) * (size_t)n * 2 * NP));
        CUDA_TRY(cudaMalloc(&X->d_g_off[s], sizeof(long long) * off.size()));
        CUDA_TRY(cudaMalloc(&X->d_g_cell[s], sizeof(long long) * std::max<size_t>(touched.size(), 1)));
        CUDA_TRY(cudaMalloc(&X->d_g_src[s], sizeof(long long) * std::max<size_t>(flat.size(), 1)));
        CUDA_TRY(cudaMemcpy(X->d_g_off[s], off.data(), sizeof(long long) * off.size(), cudaMemcpyHostToDevice));
        if (!touched.empty())
            CUDA_TRY(cudaMemcpy(X->d_g_cell[s], touched.data(), sizeof(long long) * touched.size(), cudaMemcpyHostToDevice));
        if (!flat.empty())
            CUDA_TRY(cudaMemcpy(X->d_g_src[s], flat.data(), sizeof(long long) * flat.size(), cudaMemcpyHostToDevice));
    }
    CUDA_TRY(cudaMemcpy(X->d_nodes[s], X->nodes[s].data(), sizeof(double) * 3 * nn, cudaMemcpyHostToDevice));
    double* d_mom = nullptr;
    int* d_deg = nullptr;
    double* d_res = nullptr;
    CUDA_TRY(cudaMalloc(&d_mom, sizeof(double) * XDG_MAXM * n));
    CUDA_TRY(cudaMalloc(&d_deg, sizeof(int) * n));
    CUDA_TRY(cudaMalloc(&d_res, sizeof(double) * n));
    Sub sub{};
    sub.S1 = xo.subdivision;
    sub.S2 = xo.subdivision;
    std::vector<double> gx, gw;
    gauss(3, gx, gw);
    for (int q = 0; q < 3; ++q) {
        sub.gx[q] = gx[q];
        sub.gw[q] = gw[q];
    }
    k_moments<<<n, 256>>>(X->d_items[s], n, X->ls, sub, d_mom);
    CUDA_TRY(cudaGetLastError());
    if (!saye) {
        k_weight_solve<<<n, 128>>>(X->d_items[s], n, X->d_nodes[s], d_mom, X->d_weights[s], d_deg, d_res);
        CUDA_TRY(cudaGetLastError());
    }
    CUDA_TRY(cudaDeviceSynchronize());
    X->moments[s].assign((size_t)XDG_MAXM * n, 0.0);
    CUDA_TRY(cudaMemcpy(X->moments[s].data(), d_mom, sizeof(double) * XDG_MAXM * n, cudaMemcpyDeviceToHost));
    if (saye) {
        // the rule's residual against the integrated moments: || Phi w - b || / || b ||
        if (nn) CUDA_TRY(cudaMemcpy(X->d_weights[s], X->weights[s].data(), sizeof(double) * nn, cudaMemcpyHostToDevice));
        for (int r = 0; r < n; ++r) {
            const CutItem& it = items[r];
            const int M = it.dim == 3 ? nmodes3(it.p) : nmodes2(it.p);
            double acc[XDG_MAXM] = {0.0}, v[XDG_MAXM];
            for (int q = 0; q < it.nnodes; ++q) {
                const double* xi = &X->nodes[s][(it.node_off + q) * 3];
                if (it.dim == 3) basis3(it.p, xi, v);
                else basis2(it.p, xi, v);
                for (int m = 0; m < M; ++m) acc[m] += X->weights[s][it.node_off + q] * v[m];
            }
            double num = 0.0, den = 0.0;
            for (int m = 0; m < M; ++m) {
                const double b = X->moments[s][(size_t)r * XDG_MAXM + m];
                num += (acc[m] - b) * (acc[m] - b);
                den += b * b;
            }
            // relative to the moments, floored at 1e-10 of the reference measure: sliver parts
            // whose subdivided moments vanish would otherwise divide by zero
            X->fit_resid[s][r] = std::sqrt(num) / std::max(std::sqrt(den), 1e-10);
            X->fitted_deg[s][r] = it.p;
        }
    } else {
        CUDA_TRY(cudaMemcpy(X->weights[s].data(), X->d_weights[s], sizeof(double) * nn, cudaMemcpyDeviceToHost));
        CUDA_TRY(cudaMemcpy(X->fitted_deg[s].data(), d_deg, sizeof(int) * n, cudaMemcpyDeviceToHost));
        CUDA_TRY(cudaMemcpy(X->fit_resid[s].data(), d_res, sizeof(double) * n, cudaMemcpyDeviceToHost));
    }
    cudaFree(d_mom);
    cudaFree(d_deg);
    cudaFree(d_res);
    return BOSSS_OK;
}

// Surface rules of the sphere in every cut cell (height-function quadrature, sphere_surface_box):
// cells, node offsets (cells + 1), nodes in reference coordinates of the cell (3 per node),
// weights (physical surface measure) and unit normals (3 per node).
static void surface_rules(const bosss_xdg* X, int nodes_1d, std::vector<long long>& cells, std::vector<long long>& off,
                          std::vector<double>& xi, std::vector<double>& w, std::vector<double>& nr) {
    std::vector<double> gx, gw, tmp;
    gauss(nodes_1d, gx, gw);
    const GridConst& g = X->h[0]->base.g;
    cells.clear();
    off.assign(1, 0);
    xi.clear();
    w.clear();
    nr.clear();
    const double c[3] = {X->ls.c[0], X->ls.c[1], X->ls.c[2]};
    for (int i = 0; i < g.n[0]; ++i)
        for (int j = 0; j < g.n[1]; ++j)
            for (int k = 0; k < g.n[2]; ++k) {
                const int ijk[3] = {i, j, k};
                double lo[3], hi[3];
                for (int d = 0; d < 3; ++d) {
                    lo[d] = g.lo[d] + ijk[d] * g.h[d];
                    hi[d] = lo[d] + g.h[d];
                }
                if (ls_box(X->ls, lo, hi, 7) != 0) continue;
                tmp.clear();
                sphere_surface_box(lo, hi, c, X->ls.r, gx, gw, 0, tmp);
                if (tmp.empty()) continue;
                const size_t nn = tmp.size() / 7;
                for (size_t q = 0; q < nn; ++q) {
                    for (int d = 0; d < 3; ++d) xi.push_back(2.0 * (tmp[7 * q + d] - lo[d]) / g.h[d] - 1.0);
                    w.push_back(tmp[7 * q + 3]);
                    for (int d = 0; d < 3; ++d) nr.push_back(tmp[7 * q + 4 + d]);
                }
                cells.push_back((long long)i * g.stride[0] + (long long)j * g.stride[1] + (long long)k * g.stride[2]);
                off.push_back(off.back() + (long long)nn);
            }
}

// The species' cell length scales without agglomeration, as MultiphaseAgglomerator.LengthScaleAgg
// computes them from the cut-cell metrics (MultiphaseAgglomerator.cs:744-944): for each cell of the
// species, len = V / S with V = the species volume in the cell and S = the interface area in the
// cell plus the species' part of every face of the cell (boundary faces included); len >=
// machine epsilon * h_min; with no agglomeration, cells whose volume fraction is <= 1e-10 get
// 1e10 times the uncut cell length scale. V and the face parts come from the fitted rules (the
// uncut ones are the whole cell / face), the interface area from the surface rules. Cells
// without the species get NaN (no term reads them).
static void default_length_scales(const bosss_xdg* X, int s, const std::vector<double>& iface_area,
                                  std::vector<double>& len) {
    const GridConst& g = X->h[s]->base.g;
    const long long J = g.J;
    const double vol_cell = g.h[0] * g.h[1] * g.h[2];
    double area[3];
    for (int d = 0; d < 3; ++d) area[d] = vol_cell / g.h[d];
    std::vector<double> V(J, 0.0), fa((size_t)J * 6, 0.0);
    for (long long j = 0; j < J; ++j) {
        if (X->vol[s][j] == 1) V[j] = vol_cell;
        for (int f = 0; f < 6; ++f)
            if (X->face[s][j * 6 + f] == 1) fa[j * 6 + f] = area[f / 2];
    }
    const auto& items = X->items[s];
    const auto& w = X->weights[s];
    for (const CutItem& it : items) {
        double sw = 0.0;
        for (int q = 0; q < it.nnodes; ++q) sw += w[it.node_off + q];
        if (it.dim == 3) {
            V[it.cell] = sw * g.detJ;
        } else {
            const double a = sw * g.faceSG[it.dir];
            fa[it.cell * 6 + 2 * it.dir + it.side] = a;
            int ijk[3];
            for (int d = 0; d < 3; ++d) ijk[d] = (int)((it.cell / g.stride[d]) % g.n[d]);
            const int n2 = ijk[it.dir] + (it.side ? 1 : -1);
            if (n2 >= 0 && n2 < g.n[it.dir]) {
                const long long nb = it.cell + (it.side ? 1 : -1) * g.stride[it.dir];
                fa[nb * 6 + 2 * it.dir + (1 - it.side)] = a;
            } else if (g.periodic[it.dir]) {
                const long long nb = it.cell + (long long)(it.side ? -(g.n[it.dir] - 1) : (g.n[it.dir] - 1)) * g.stride[it.dir];
                fa[nb * 6 + 2 * it.dir + (1 - it.side)] = a;
            }
        }
    }
    const double hmin = std::min(g.h[0], std::min(g.h[1], g.h[2]));
    len.assign(J, std::nan(""));
    for (long long j = 0; j < J; ++j) {
        if (X->vol[s][j] == 0) continue;
        double S = iface_area[j];
        for (int f = 0; f < 6; ++f) S += fa[j * 6 + f];
        double L = std::nan("");
        if (std::fabs(S) >= 1e-25) L = std::max(V[j] / S, 2.220446049250313e-16 * hmin);
        if (V[j] / vol_cell <= 1e-10) {
            // the reference's treatment of vanishing fractions without agglomeration
            int ijk[3];
            double cj = 0.0;
            for (int d = 0; d < 3; ++d) {
                ijk[d] = (int)((j / g.stride[d]) % g.n[d]);
                const int nb = g.periodic[d] ? 0 : (ijk[d] == 0) + (ijk[d] == g.n[d] - 1);
                cj += (2.0 + nb) / g.h[d];
            }
            L = 1e10 / (0.5 * cj);
        }
        len[j] = L;
    }
}

// upload 1/len of species s and point the species' handles at it
static int apply_length_scales(bosss_xdg* X, int s) {
    const long long J = (long long)X->len[s].size();
    std::vector<double> pf(J);
    for (long long j = 0; j < J; ++j) {
        const double L = X->len[s][j];
        pf[j] = (std::isfinite(L) && L > 0.0) ? 1.0 / L : 0.0;
    }
    CUDA_TRY(cudaSetDevice(X->device));
    if (!X->d_pf[s]) CUDA_TRY(cudaMalloc(&X->d_pf[s], sizeof(double) * std::max<long long>(J, 1)));
    CUDA_TRY(cudaMemcpy(X->d_pf[s], pf.data(), sizeof(double) * J, cudaMemcpyHostToDevice));
    X->h[s]->base.cell_pf = X->d_pf[s];
    if (s == 1 && X->hs) X->hs->base.cell_pf = X->d_pf[s];
    X->ifa.pfA = X->d_pf[0];
    X->ifa.pfB = X->d_pf[1];
    return BOSSS_OK;
}

}  // namespace bosss

extern "C" {

int bosss_b200_xdg_create(const bosss_op_desc* opA, const bosss_op_desc* opB, const bosss_grid_desc* grid,
                          const bosss_levelset_desc* ls, const bosss_xdg_opts* xopt, const bosss_options* opt,
                          bosss_xdg** out) {
    if (!opA || !opB || !grid || !ls || !out) return fail(BOSSS_ERR_BAD_ARG, "null argument");
    *out = nullptr;
    if (grid->dim != 3) return fail(BOSSS_ERR_BAD_ARG, "XDG path: 3D grids");
    if (ls->type != BOSSS_LEVELSET_SPHERE || !(ls->params[3] > 0.0))
        return fail(BOSSS_ERR_BAD_ARG, "XDG path: sphere level set phi = |x - c| - r, r > 0");
    bosss_xdg_opts xo{};
    xo.cut_nodes_1d = 5;
    xo.fallback_nodes_1d = 9;
    xo.moment_degree = -1;
    xo.subdivision = 8;
    if (xopt) {
        if (xopt->cut_nodes_1d > 0) xo.cut_nodes_1d = xopt->cut_nodes_1d;
        if (xopt->fallback_nodes_1d > 0) xo.fallback_nodes_1d = xopt->fallback_nodes_1d;
        if (xopt->moment_degree >= 0) xo.moment_degree = xopt->moment_degree;
        if (xopt->subdivision > 0) xo.subdivision = xopt->subdivision;
        xo.rule = xopt->rule;
    }
    if (xo.rule != 0 && xo.rule != 1) return fail(BOSSS_ERR_BAD_ARG, "XDG rule family: 0 or 1");
    // the species masks of the bulk evaluation are read by the generic and the slab kernels
    bosss_options hopt{};
    if (opt) hopt = *opt;
    if (hopt.kernel == 3) return fail(BOSSS_ERR_BAD_ARG, "XDG evaluation: kernel 0, 1 or 2");
    if (hopt.precision != BOSSS_PRECISION_FP64) return fail(BOSSS_ERR_BAD_ARG, "XDG evaluation runs in FP64");
    bosss_xdg* X = new bosss_xdg();
    for (int s = 0; s < 2; ++s) {
        int rc = bosss_b200_create(s == 0 ? opA : opB, grid, &hopt, &X->h[s]);
        if (rc) {
            bosss_b200_xdg_destroy(X);
            return rc;
        }
        if (X->h[s]->phys != PHYS_SIP || X->h[s]->D != 3 || X->h[s]->K < 1 || X->h[s]->K > 4) {
            bosss_b200_xdg_destroy(X);
            return fail(BOSSS_ERR_UNSUPPORTED_COMPONENT, "XDG bulk: SIP (XLaplace_Bulk) operators, degree 1..4");
        }
    }
    X->device = X->h[0]->device;
    X->K = X->h[0]->K;
    if (X->h[1]->K != X->K) {
        bosss_b200_xdg_destroy(X);
        return fail(BOSSS_ERR_BAD_ARG, "both species need the same DG degree");
    }
    if (xo.moment_degree < 0) xo.moment_degree = std::min(4, 2 * X->K);
    if (xo.moment_degree > 4) xo.moment_degree = 4;
    X->ls.type = ls->type;
    for (int d = 0; d < 3; ++d) X->ls.c[d] = ls->params[d];
    X->ls.r = ls->params[3];
    cudaError_t e = cudaSetDevice(X->device);
    if (e != cudaSuccess) {
        bosss_b200_xdg_destroy(X);
        return fail(BOSSS_ERR_CUDA, cudaGetErrorString(e));
    }
    for (int s = 0; s < 2; ++s) {
        int rc = build_species(X, s, xo);
        if (!rc) rc = upload_and_fit(X, s, xo);
        if (rc) {
            bosss_b200_xdg_destroy(X);
            return rc;
        }
        long long j0 = -1, j1 = 0;
        for (long long j = 0; j < (long long)X->vol[s].size(); ++j)
            if (X->vol[s][j] != 0) {
                if (j0 < 0) j0 = j;
                j1 = j + 1;
            }
        X->rng[s][0] = j0 < 0 ? 0 : j0;
        X->rng[s][1] = j1;
        if (s == 1) {
            // planes of species B holding a cell that is not plain species B
            const long long J = (long long)X->vol[1].size(), P = X->h[1]->base.g.stride[0];
            long long b0 = J, b1 = 0;
            for (long long j = 0; j < J; ++j) {
                bool plain = X->vol[1][j] == 1;
                for (int f = 0; f < 6 && plain; ++f) plain = X->face[1][j * 6 + f] == 1;
                if (!plain) {
                    b0 = std::min(b0, j);
                    b1 = j + 1;
                }
            }
            if (b1 <= b0) b0 = b1 = 0;
            X->sb[0] = (b0 / P) * P;
            X->sb[1] = std::min(J, ((b1 + P - 1) / P) * P);
            bosss_options sopt = hopt;
            sopt.kernel = 2;
            if (X->sb[1] - X->sb[0] < J && bosss_b200_create(opB, grid, &sopt, &X->hs) != BOSSS_OK) X->hs = nullptr;
        }
    }
    {
        // default cell length scales of both species (interface areas from the surface rules)
        std::vector<long long> cells, off;
        std::vector<double> xi, w, nr;
        surface_rules(X, 6, cells, off, xi, w, nr);
        std::vector<double> ia((size_t)X->h[0]->base.g.J, 0.0);
        for (size_t r = 0; r < cells.size(); ++r)
            for (long long q = off[r]; q < off[r + 1]; ++q) ia[cells[r]] += w[q];
        for (int s = 0; s < 2; ++s) {
            default_length_scales(X, s, ia, X->len_default[s]);
            X->len[s] = X->len_default[s];
            const int rc = apply_length_scales(X, s);
            if (rc) {
                bosss_b200_xdg_destroy(X);
                return rc;
            }
        }
    }
    *out = X;
    return BOSSS_OK;
}

int bosss_b200_xdg_get_length_scales(const bosss_xdg* X, int32_t species, double* len) {
    if (!X || species < 0 || species > 1 || !len) return fail(BOSSS_ERR_BAD_ARG, "bad argument");
    std::copy(X->len[species].begin(), X->len[species].end(), len);
    return BOSSS_OK;
}

int bosss_b200_xdg_set_length_scales(bosss_xdg* X, int32_t species, const double* len) {
    if (!X || species < 0 || species > 1) return fail(BOSSS_ERR_BAD_ARG, "bad argument");
    const long long J = (long long)X->len_default[species].size();
    if (len) {
        for (long long j = 0; j < J; ++j)
            if (X->vol[species][j] != 0 && !(std::isfinite(len[j]) && len[j] > 0.0))
                return fail(BOSSS_ERR_BAD_ARG, "length scales of the species' cells must be finite and positive (cell " +
                                                   std::to_string(j) + ")");
        X->len[species].assign(len, len + J);
    } else {
        X->len[species] = X->len_default[species];
    }
    return apply_length_scales(X, species);
}

int bosss_b200_saye_rule(const bosss_levelset_desc* ls, int32_t dim, int32_t dir, int32_t species,
                         const double* center, const double* h, int32_t nodes_1d, int64_t* n_nodes, double* nodes,
                         double* weights) {
    if (!ls || !center || !h || !n_nodes) return fail(BOSSS_ERR_BAD_ARG, "null argument");
    if (ls->type != BOSSS_LEVELSET_SPHERE || !(ls->params[3] > 0.0))
        return fail(BOSSS_ERR_BAD_ARG, "Saye rule: sphere level set phi = |x - c| - r, r > 0");
    if ((dim != 2 && dim != 3) || dir < 0 || dir > 2 || (species != -1 && species != 1) || nodes_1d < 1 ||
        nodes_1d > 16)
        return fail(BOSSS_ERR_BAD_ARG, "Saye rule: dim 2 or 3, dir 0..2, species -1 or +1, 1..16 nodes");
    for (int d = 0; d < 3; ++d)
        if (!(h[d] > 0.0)) return fail(BOSSS_ERR_BAD_ARG, "Saye rule: positive cell size");
    LevelSetDev L{};
    L.type = ls->type;
    for (int d = 0; d < 3; ++d) L.c[d] = ls->params[d];
    L.r = ls->params[3];
    CutItem it{};
    it.dim = dim;
    it.dir = dir;
    it.sp = species;
    for (int d = 0; d < 3; ++d) {
        it.center[d] = center[d];
        it.h[d] = h[d];
    }
    std::vector<double> gx, gw, nd, wt;
    gauss(nodes_1d, gx, gw);
    const int n = saye_item_rule(L, it, gx, gw, nd, wt);
    if (nodes && weights) {
        if (*n_nodes < n) return fail(BOSSS_ERR_BAD_ARG, "Saye rule: arrays too small");
        std::memcpy(nodes, nd.data(), sizeof(double) * nd.size());
        std::memcpy(weights, wt.data(), sizeof(double) * wt.size());
    }
    *n_nodes = n;
    return BOSSS_OK;
}

int bosss_b200_xdg_destroy(bosss_xdg* X) {
    if (!X) return BOSSS_OK;
    cudaSetDevice(X->device);
    for (int s = 0; s < 2; ++s) cudaFree(X->d_pf[s]);
    for (int s = 0; s < 2; ++s) {
        cudaFree(X->d_vol[s]);
        cudaFree(X->d_face[s]);
        cudaFree(X->d_items[s]);
        cudaFree(X->d_item_out[s]);
        cudaFree(X->d_g_off[s]);
        cudaFree(X->d_g_cell[s]);
        cudaFree(X->d_g_src[s]);
        cudaFree(X->d_nodes[s]);
        cudaFree(X->d_weights[s]);
        bosss_b200_destroy(X->h[s]);
    }
    bosss_b200_destroy(X->hs);
    cudaFree(X->d_if_cells);
    cudaFree(X->d_if_off);
    cudaFree(X->d_if_nodes);
    cudaFree(X->d_if_w);
    cudaFree(X->d_if_n);
    delete X;
    return BOSSS_OK;
}

int bosss_b200_xdg_info(const bosss_xdg* X, int32_t species, int64_t* n_cells, int64_t* n_cut_cells,
                        int64_t* n_cut_faces, int32_t* min_nodes, int32_t* max_nodes, int32_t* min_degree,
                        double* max_fit_residual) {
    if (!X || species < 0 || species > 1) return fail(BOSSS_ERR_BAD_ARG, "bad argument");
    const int s = species;
    long long nc = 0, nf = 0;
    int mn = 1 << 30, mx = 0, mdeg = 99;
    double r = 0.0;
    for (size_t i = 0; i < X->items[s].size(); ++i) {
        const CutItem& it = X->items[s][i];
        (it.dim == 3 ? nc : nf)++;
        mn = std::min(mn, it.nnodes);
        mx = std::max(mx, it.nnodes);
        mdeg = std::min(mdeg, X->fitted_deg[s][i]);
        r = std::max(r, X->fit_resid[s][i]);
    }
    if (n_cells) *n_cells = X->n_cells[s];
    if (n_cut_cells) *n_cut_cells = nc;
    if (n_cut_faces) *n_cut_faces = nf;
    if (min_nodes) *min_nodes = X->items[s].empty() ? 0 : mn;
    if (max_nodes) *max_nodes = mx;
    if (min_degree) *min_degree = X->items[s].empty() ? -1 : mdeg;
    if (max_fit_residual) *max_fit_residual = r;
    return BOSSS_OK;
}

int bosss_b200_xdg_get_rules(const bosss_xdg* X, int32_t species, int64_t* n_items, int64_t* item_info,
                             int64_t* node_offsets, double* nodes, double* weights, unsigned char* vol_flags,
                             unsigned char* face_flags) {
    if (!X || species < 0 || species > 1) return fail(BOSSS_ERR_BAD_ARG, "bad argument");
    const int s = species;
    const auto& items = X->items[s];
    if (n_items) n_items[0] = (int64_t)items.size(), n_items[1] = (int64_t)(X->nodes[s].size() / 3);
    for (size_t i = 0; i < items.size(); ++i) {
        if (item_info) {
            item_info[i * 5 + 0] = items[i].cell;
            item_info[i * 5 + 1] = items[i].dim;
            item_info[i * 5 + 2] = items[i].dir;
            item_info[i * 5 + 3] = items[i].side;
            item_info[i * 5 + 4] = X->fitted_deg[s][i];
        }
        if (node_offsets) node_offsets[i] = items[i].node_off;
    }
    if (node_offsets) node_offsets[items.size()] = (int64_t)(X->nodes[s].size() / 3);
    if (nodes) std::memcpy(nodes, X->nodes[s].data(), sizeof(double) * X->nodes[s].size());
    if (weights) std::memcpy(weights, X->weights[s].data(), sizeof(double) * X->weights[s].size());
    if (vol_flags) std::memcpy(vol_flags, X->vol[s].data(), X->vol[s].size());
    if (face_flags) std::memcpy(face_flags, X->face[s].data(), X->face[s].size());
    return BOSSS_OK;
}

int bosss_b200_xdg_get_moments(const bosss_xdg* X, int32_t species, double* moments) {
    if (!X || species < 0 || species > 1 || !moments) return fail(BOSSS_ERR_BAD_ARG, "bad argument");
    std::memcpy(moments, X->moments[species].data(), sizeof(double) * X->moments[species].size());
    return BOSSS_OK;
}

int bosss_b200_xdg_evaluate_device(bosss_xdg* X, int32_t species, double alpha, double beta, const double* U_dev,
                                   double* out_dev, double time, void* stream) {
    if (!X || species < 0 || species > 1 || !U_dev || !out_dev) return fail(BOSSS_ERR_BAD_ARG, "bad argument");
    const int s = species;
    bosss_handle* h = X->h[s];
    CUDA_TRY(cudaSetDevice(X->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
    // uncut cells and faces of the species: tensor kernel with masks
    // only the band of cells holding the species is launched; the others get out = beta * out
    const long long c0 = X->rng[s][0], c1 = X->rng[s][1], NP = np_of(3, X->K), J = h->base.g.J;
    if (beta != 1.0) {
        for (int part = 0; part < 2; ++part) {
            const long long a0 = part ? c1 * NP : 0, a1 = part ? J * NP : c0 * NP;
            if (a1 <= a0) continue;
            if (beta == 0.0) {
                CUDA_TRY(cudaMemsetAsync(out_dev + a0, 0, sizeof(double) * (a1 - a0), st));
            } else {
                k_scale<<<592, 256, 0, st>>>(out_dev + a0, a1 - a0, beta);
                CUDA_TRY(cudaGetLastError());
            }
        }
    }
    int rc = 0;
    // species B: the planes of plain species-B cells go to the unmasked slab kernel
    const bool split = (s == 1 && X->hs != nullptr);
    const long long m0 = split ? std::max(c0, X->sb[0]) : c0, m1 = split ? std::min(c1, X->sb[1]) : c1;
    if (m1 > m0) {
        EvalArgs keep = h->base;
        h->base.vol_flag = X->d_vol[s];
        h->base.face_flag = X->d_face[s];
        h->base.cbeg = m0;
        h->base.cend = m1;
        rc = run_mode(h, MODE_RES, alpha, beta, U_dev, nullptr, out_dev, time, st);
        h->base = keep;
    }
    if (rc) return rc;
    if (split) {
        const long long parts[2][2] = {{c0, std::min(c1, X->sb[0])}, {std::max(c0, X->sb[1]), c1}};
        for (int part = 0; part < 2; ++part) {
            if (parts[part][1] <= parts[part][0]) continue;
            rc = bosss_b200_apply_device(X->hs, MODE_RES, alpha, beta, U_dev, nullptr, out_dev, time,
                                         parts[part][0], parts[part][1], st);
            if (rc) return rc;
        }
    }
    // cut cells and faces: explicit rules, added atomically
    const int n = (int)X->items[s].size();
    if (n > 0) {
        EvalArgs a = h->base;
        a.U = U_dev;
        a.out = out_dev;
        a.alpha = alpha;
        a.time = time;
        switch (X->K) {
            case 1: k_cut_eval<1><<<n, 64, 0, st>>>(X->d_items[s], n, X->d_nodes[s], X->d_weights[s], a, X->d_item_out[s]); break;
            case 2: k_cut_eval<2><<<n, 64, 0, st>>>(X->d_items[s], n, X->d_nodes[s], X->d_weights[s], a, X->d_item_out[s]); break;
            case 3: k_cut_eval<3><<<n, 64, 0, st>>>(X->d_items[s], n, X->d_nodes[s], X->d_weights[s], a, X->d_item_out[s]); break;
            default: k_cut_eval<4><<<n, 64, 0, st>>>(X->d_items[s], n, X->d_nodes[s], X->d_weights[s], a, X->d_item_out[s]); break;
        }
        CUDA_TRY(cudaGetLastError());
        const long long nc = X->n_gcells[s], NPc = np_of(3, X->K);
        const int gg = (int)std::max<long long>(1, std::min<long long>((nc * NPc + 255) / 256, 148LL * 16));
        switch (X->K) {
            case 1: k_cut_gather<1><<<gg, 256, 0, st>>>(nc, X->d_g_off[s], X->d_g_cell[s], X->d_g_src[s], X->d_item_out[s], out_dev); break;
            case 2: k_cut_gather<2><<<gg, 256, 0, st>>>(nc, X->d_g_off[s], X->d_g_cell[s], X->d_g_src[s], X->d_item_out[s], out_dev); break;
            case 3: k_cut_gather<3><<<gg, 256, 0, st>>>(nc, X->d_g_off[s], X->d_g_cell[s], X->d_g_src[s], X->d_item_out[s], out_dev); break;
            default: k_cut_gather<4><<<gg, 256, 0, st>>>(nc, X->d_g_off[s], X->d_g_cell[s], X->d_g_src[s], X->d_item_out[s], out_dev); break;
        }
        CUDA_TRY(cudaGetLastError());
    }
    return BOSSS_OK;
}

int bosss_b200_xdg_evaluate(bosss_xdg* X, int32_t species, double alpha, double beta, const double* U, double* out,
                            double time) {
    if (!X || species < 0 || species > 1 || !U || !out) return fail(BOSSS_ERR_BAD_ARG, "bad argument");
    bosss_handle* h = X->h[species];
    int rc = ensure_staging(h);
    if (rc) return rc;
    CUDA_TRY(cudaSetDevice(X->device));
    cudaStream_t s = h->stream;
    CUDA_TRY(cudaMemcpyAsync(h->dU, U, sizeof(double) * h->ndom, cudaMemcpyHostToDevice, s));
    if (beta != 0.0) CUDA_TRY(cudaMemcpyAsync(h->dOut, out, sizeof(double) * h->ncod, cudaMemcpyHostToDevice, s));
    rc = bosss_b200_xdg_evaluate_device(X, species, alpha, beta, h->dU, h->dOut, time, s);
    if (rc) return rc;
    CUDA_TRY(cudaMemcpyAsync(out, h->dOut, sizeof(double) * h->ncod, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    return BOSSS_OK;
}


// ---- level-set interface term: XLaplace_Interface on the sphere surface (NECQuadratureLevelSet)
int bosss_b200_xdg_interface_setup(bosss_xdg* X, double mu_A, double mu_B, double penalty_base, int32_t mode,
                                   int32_t nodes_1d) {
    if (!X) return fail(BOSSS_ERR_BAD_ARG, "null handle");
    if (mode != BOSSS_IFACE_SWIP && mode != BOSSS_IFACE_SIP) return fail(BOSSS_ERR_BAD_ARG, "mode: SWIP (0) or SIP (1)");
    // ComputeScaling asserts sign(muA) == sign(muB) (XLaplace.cs:302-322)
    if (!(mu_A * mu_B > 0.0) || !std::isfinite(mu_A) || !std::isfinite(mu_B))
        return fail(BOSSS_ERR_BAD_ARG, "mu_A and mu_B must be finite, nonzero and of the same sign");
    if (!std::isfinite(penalty_base)) return fail(BOSSS_ERR_BAD_ARG, "penalty_base must be finite");
    if (nodes_1d <= 0) nodes_1d = 6;
    if (nodes_1d > 16) return fail(BOSSS_ERR_BAD_ARG, "nodes_1d: 1..16");
    const int K = X->K;
    IfaceArgs f{};
    f.muA = mu_A;
    f.muB = mu_B;
    double pen_mu;
    if (mode == BOSSS_IFACE_SWIP) {
        f.omA = mu_B / (mu_A + mu_B);
        f.omB = mu_A / (mu_A + mu_B);
        pen_mu = 2.0 * mu_A * mu_B / (mu_A + mu_B);
    } else {
        f.omA = 0.5;
        f.omB = 0.5;
        pen_mu = std::max(std::fabs(mu_A), std::fabs(mu_B)) * (mu_A > 0.0 ? 1.0 : -1.0);
    }
    // CoefficientUpdate (XLaplace.cs:331-341): max of the simplex and the cube formula, D = 3
    const double pdeg = std::max((K + 1.0) * (K + 3.0) / 3.0, (K + 1.0) * (K + 1.0));
    f.pen = penalty_base * pdeg * pen_mu;
    f.alpha = 1.0;
    std::vector<long long> cells, off;
    std::vector<double> xi, w, nr;
    surface_rules(X, nodes_1d, cells, off, xi, w, nr);
    f.pfA = X->d_pf[0];
    f.pfB = X->d_pf[1];
    CUDA_TRY(cudaSetDevice(X->device));
    cudaFree(X->d_if_cells);
    cudaFree(X->d_if_off);
    cudaFree(X->d_if_nodes);
    cudaFree(X->d_if_w);
    cudaFree(X->d_if_n);
    X->d_if_cells = nullptr;
    X->d_if_off = nullptr;
    X->d_if_nodes = X->d_if_w = X->d_if_n = nullptr;
    X->iface = false;
    const size_t nc = cells.size(), nq = w.size();
    CUDA_TRY(cudaMalloc(&X->d_if_cells, sizeof(long long) * std::max<size_t>(nc, 1)));
    CUDA_TRY(cudaMalloc(&X->d_if_off, sizeof(long long) * (nc + 1)));
    CUDA_TRY(cudaMalloc(&X->d_if_nodes, sizeof(double) * 3 * std::max<size_t>(nq, 1)));
    CUDA_TRY(cudaMalloc(&X->d_if_w, sizeof(double) * std::max<size_t>(nq, 1)));
    CUDA_TRY(cudaMalloc(&X->d_if_n, sizeof(double) * 3 * std::max<size_t>(nq, 1)));
    if (nc) CUDA_TRY(cudaMemcpy(X->d_if_cells, cells.data(), sizeof(long long) * nc, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(X->d_if_off, off.data(), sizeof(long long) * (nc + 1), cudaMemcpyHostToDevice));
    if (nq) {
        CUDA_TRY(cudaMemcpy(X->d_if_nodes, xi.data(), sizeof(double) * 3 * nq, cudaMemcpyHostToDevice));
        CUDA_TRY(cudaMemcpy(X->d_if_w, w.data(), sizeof(double) * nq, cudaMemcpyHostToDevice));
        CUDA_TRY(cudaMemcpy(X->d_if_n, nr.data(), sizeof(double) * 3 * nq, cudaMemcpyHostToDevice));
    }
    X->if_cells.swap(cells);
    X->if_off.swap(off);
    X->if_nodes.swap(xi);
    X->if_w.swap(w);
    X->if_n.swap(nr);
    X->ifa = f;
    X->iface = true;
    return BOSSS_OK;
}

int bosss_b200_xdg_interface_get_rules(const bosss_xdg* X, int64_t* counts, int64_t* cells, int64_t* node_offsets,
                                       double* nodes, double* weights, double* normals) {
    if (!X || !counts) return fail(BOSSS_ERR_BAD_ARG, "null argument");
    if (!X->iface) return fail(BOSSS_ERR_BAD_ARG, "interface term not set up (bosss_b200_xdg_interface_setup)");
    const size_t nc = X->if_cells.size(), nq = X->if_w.size();
    counts[0] = (int64_t)nc;
    counts[1] = (int64_t)nq;
    if (cells) for (size_t i = 0; i < nc; ++i) cells[i] = X->if_cells[i];
    if (node_offsets) for (size_t i = 0; i <= nc; ++i) node_offsets[i] = X->if_off[i];
    if (nodes) std::memcpy(nodes, X->if_nodes.data(), sizeof(double) * 3 * nq);
    if (weights) std::memcpy(weights, X->if_w.data(), sizeof(double) * nq);
    if (normals) std::memcpy(normals, X->if_n.data(), sizeof(double) * 3 * nq);
    return BOSSS_OK;
}

int bosss_b200_xdg_interface_evaluate_device(bosss_xdg* X, double alpha, const double* UA_dev, const double* UB_dev,
                                             double* outA_dev, double* outB_dev, void* stream) {
    if (!X || !UA_dev || !UB_dev || !outA_dev || !outB_dev) return fail(BOSSS_ERR_BAD_ARG, "null argument");
    if (!X->iface) return fail(BOSSS_ERR_BAD_ARG, "interface term not set up (bosss_b200_xdg_interface_setup)");
    CUDA_TRY(cudaSetDevice(X->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : X->h[0]->stream;
    const int n = (int)X->if_cells.size();
    if (n == 0) return BOSSS_OK;
    IfaceArgs f = X->ifa;
    f.alpha = alpha;
    const GridConst& g = X->h[0]->base.g;
    switch (X->K) {
#define BOSSS_IFACE_LAUNCH(KK)                                                                                  \
    case KK:                                                                                                    \
        k_interface_eval<KK><<<n, 64, 0, st>>>(X->d_if_cells, X->d_if_off, X->d_if_nodes, X->d_if_w, X->d_if_n, \
                                               n, g, f, UA_dev, UB_dev, outA_dev, outB_dev);                   \
        break;
        BOSSS_IFACE_LAUNCH(1)
        BOSSS_IFACE_LAUNCH(2)
        BOSSS_IFACE_LAUNCH(3)
        BOSSS_IFACE_LAUNCH(4)
#undef BOSSS_IFACE_LAUNCH
        default: return fail(BOSSS_ERR_BAD_ARG, "degree 1..4");
    }
    CUDA_TRY(cudaGetLastError());
    return BOSSS_OK;
}

int bosss_b200_xdg_interface_evaluate(bosss_xdg* X, double alpha, const double* UA, const double* UB, double* outA,
                                      double* outB) {
    if (!X || !UA || !UB || !outA || !outB) return fail(BOSSS_ERR_BAD_ARG, "null argument");
    if (!X->iface) return fail(BOSSS_ERR_BAD_ARG, "interface term not set up (bosss_b200_xdg_interface_setup)");
    CUDA_TRY(cudaSetDevice(X->device));
    const size_t nb = sizeof(double) * (size_t)X->h[0]->ncod;
    double* buf = nullptr;
    CUDA_TRY(cudaMalloc(&buf, 4 * nb));
    double *dUA = buf, *dUB = buf + X->h[0]->ncod, *dA = buf + 2 * X->h[0]->ncod, *dB = buf + 3 * X->h[0]->ncod;
    cudaStream_t st = X->h[0]->stream;
    cudaError_t e = cudaMemcpyAsync(dUA, UA, nb, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dUB, UB, nb, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dA, outA, nb, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dB, outB, nb, cudaMemcpyHostToDevice, st);
    int rc = BOSSS_OK;
    if (e == cudaSuccess) rc = bosss_b200_xdg_interface_evaluate_device(X, alpha, dUA, dUB, dA, dB, st);
    if (e == cudaSuccess && rc == BOSSS_OK) e = cudaMemcpyAsync(outA, dA, nb, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && rc == BOSSS_OK) e = cudaMemcpyAsync(outB, dB, nb, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(buf);
    if (rc) return rc;
    if (e != cudaSuccess) return fail(BOSSS_ERR_CUDA, cudaGetErrorString(e));
    return BOSSS_OK;
}

}  // extern "C"
