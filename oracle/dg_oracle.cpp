// dg_oracle.cpp -- CPU FP64 restatement of BoSSS's nonlinear DG operator evaluation.
//
// TEST INFRASTRUCTURE ONLY. This file is the oracle that the GPU path is checked
// against; it is loaded by the tests, by __graft_entry__.smoke() and by bench.py's
// CPU-baseline leg, never by the product library.
//
// It restates, for uniform affine Cartesian grids, the algorithm of
//   EvaluatorNonLin.Evaluate            DifferentialOperator.cs:1584-1661
//   NECQuadratureVolume.EvaluateEx      NECQuadratureVolume.cs:328-750 (+ SaveIntegrationResults :767-798)
//   NECQuadratureEdge.EvaluateEx        NECQuadratureEdge.cs:642-1427 (+ SaveIntegrationResults :326-412)
//   DGField.Evaluate / EvaluateGradient DGField_Evaluation.cs:38-310
//   BasisData scaling 1/sqrt(detJ)      BasisData.cs:34-60
//   cell length scale                   GridData_CellData.cs:663-698
// with the straightforward structure of the reference: basis values tabulated
// at the quadrature nodes from the monomial representation of the orthonormal
// polynomials (Square.cs:194-6481, Cube_polynomials.cs:15-13834), dense
// contractions per cell, and an edge-centric pass that scatters +IN / -OUT
// contributions to both neighbouring cells.
//
// Equation components (pointwise forms restated from the C# sources):
//   ScalarTransportFlux / ScalarTransportFlux3D   ScalarTransport/TransportFlux.cs:29-191
//   SIPLaplace                                     NSECommon/ipLaplace.cs:30-269
//   OptimizedHLLC{Density,Momentum,Energy}Flux     CompressibleFlowCommon/Convection/OptimizedHLLC*.cs
//   constant source (INonlinearSource)             NECQuadratureVolume.cs:465-489
//   OptimizedSIPG{Density,Momentum,Energy}Flux     CNS/Diffusion/OptimizedSIPG*Flux.cs (viscous
//     compressible Navier-Stokes terms, Hartmann's G tensors, Sutherland viscosity
//     MaterialProperty/SutherlandLaw.cs:25-75), with the outer boundary state prescribed per
//     boundary node (SupersonicInlet.GetBoundaryState, Boundary/SupersonicInlet.cs:45-66)
//
// The oracle is templated on the scalar type so that a forward-mode dual
// number gives the exact directional derivative (JVP) and, column by column
// over a distance-2 cell colouring, the assembled Jacobian (the analogue of
// FDJacobianBuilder, DifferentialOperator.cs:2558-2858, without the FD error).
// The adjoint product J^T W is the gradient of the functional W . Op(U): per volume
// node and per edge node the local form values are differentiated (multi-slot dual
// numbers) with respect to the node states of the cells that enter them, and chained
// back to those cells' coefficients -- the transpose of the assembled Jacobian applied
// to W, without assembling it.
//
// Pinning: the basis and Gauss-rule tables are checked against the reference's
// own tables (tests/golden/ref_*.json); the evaluator is checked against the
// DerivativeTest-style known answers (consistency on polynomial fields,
// orthonormality) in tests/test_oracle.py.

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../include/bosss_b200.h"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

// ------------------------------------------------------------------ dual numbers
struct Dual {
    double v, d;
    Dual() : v(0), d(0) {}
    Dual(double a) : v(a), d(0) {}
    Dual(double a, double b) : v(a), d(b) {}
};
inline Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
inline Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
inline Dual operator-(Dual a) { return {-a.v, -a.d}; }
inline Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
inline Dual operator/(Dual a, Dual b) { return {a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)}; }
inline Dual& operator+=(Dual& a, Dual b) { a = a + b; return a; }
inline Dual& operator-=(Dual& a, Dual b) { a = a - b; return a; }
inline Dual& operator*=(Dual& a, Dual b) { a = a * b; return a; }
inline Dual& operator/=(Dual& a, Dual b) { a = a / b; return a; }
inline bool operator>(Dual a, Dual b) { return a.v > b.v; }
inline bool operator<(Dual a, Dual b) { return a.v < b.v; }
inline bool operator>=(Dual a, Dual b) { return a.v >= b.v; }
inline bool operator<=(Dual a, Dual b) { return a.v <= b.v; }
inline Dual sqrt(Dual a) { double s = std::sqrt(a.v); return {s, a.d / (2.0 * s)}; }
inline double val(double a) { return a; }
inline double val(Dual a) { return a.v; }
using std::sqrt;
template <class T> inline T tmax(T a, T b) { return (a > b) ? a : b; }  // Math.Max semantics for finite values
template <class T> inline T tabs(T a) { return (a < T(0.0)) ? -a : a; }

// Multi-slot forward dual number: value and the derivatives with respect to N inputs. The
// operators are in-class friends (not templates), so doubles convert implicitly as for Dual.
template <int N>
struct DualV {
    double v;
    double d[N];
    DualV() : v(0) { std::memset(d, 0, sizeof(d)); }
    DualV(double a) : v(a) { std::memset(d, 0, sizeof(d)); }
    friend DualV operator+(const DualV& a, const DualV& b) {
        DualV r; r.v = a.v + b.v;
        for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
        return r;
    }
    friend DualV operator-(const DualV& a, const DualV& b) {
        DualV r; r.v = a.v - b.v;
        for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
        return r;
    }
    friend DualV operator-(const DualV& a) {
        DualV r; r.v = -a.v;
        for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
        return r;
    }
    friend DualV operator*(const DualV& a, const DualV& b) {
        DualV r; r.v = a.v * b.v;
        for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
        return r;
    }
    friend DualV operator/(const DualV& a, const DualV& b) {
        DualV r; r.v = a.v / b.v;
        const double ib2 = 1.0 / (b.v * b.v);
        for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] * b.v - a.v * b.d[i]) * ib2;
        return r;
    }
    friend DualV& operator+=(DualV& a, const DualV& b) { a = a + b; return a; }
    friend DualV& operator-=(DualV& a, const DualV& b) { a = a - b; return a; }
    friend DualV& operator*=(DualV& a, const DualV& b) { a = a * b; return a; }
    friend DualV& operator/=(DualV& a, const DualV& b) { a = a / b; return a; }
    friend bool operator>(const DualV& a, const DualV& b) { return a.v > b.v; }
    friend bool operator<(const DualV& a, const DualV& b) { return a.v < b.v; }
    friend bool operator>=(const DualV& a, const DualV& b) { return a.v >= b.v; }
    friend bool operator<=(const DualV& a, const DualV& b) { return a.v <= b.v; }
    friend DualV sqrt(const DualV& a) {
        DualV r; r.v = std::sqrt(a.v);
        const double f = 0.5 / r.v;
        for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * f;
        return r;
    }
    friend double val(const DualV& a) { return a.v; }
};

// CNS viscous components (BOSSS_COMP_CNS_SIPG_*_FLUX of the C-ABI): arguments = the D+2
// conservative variables; params[0] gamma, [1] Mach, [2] Reynolds, [3] Prandtl, [4] viscosity
// ratio (bulk/shear), [5] viscosity law (0: mu = 1, 1: Sutherland), [6] Sutherland S/T0,
// [7] SIPG penalty scaling, [8] momentum component (0-based). Boundary faces take the outer
// state from the boundary-state table (one value per domain variable and boundary face node).
enum {
    ORC_COMP_CNS_SIPG_DENSITY = BOSSS_COMP_CNS_SIPG_DENSITY_FLUX,
    ORC_COMP_CNS_SIPG_MOMENTUM = BOSSS_COMP_CNS_SIPG_MOMENTUM_FLUX,
    ORC_COMP_CNS_SIPG_ENERGY = BOSSS_COMP_CNS_SIPG_ENERGY_FLUX
};

// ------------------------------------------------------------------ basis
// Orthonormal polynomials on [-1,1]^D: products of normalised Legendre polynomials,
// ordered by total degree, then by x-exponent, then y-exponent (the order of
// Square.cs / Cube_polynomials.cs: 1, z, y, x, z^2, yz, y^2, xz, xy, x^2, ...).
struct Poly {
    std::vector<double> coef;
    std::vector<std::array<int, 3>> exps;
};

static std::vector<long double> legendre_monomials(int n) {
    // coefficients c[p] of P_n(x) = sum_p c[p] x^p, via (m+1)P_{m+1} = (2m+1) x P_m - m P_{m-1}
    std::vector<std::vector<long double>> P(n + 1, std::vector<long double>(n + 1, 0.0L));
    P[0][0] = 1.0L;
    if (n >= 1) P[1][1] = 1.0L;
    for (int m = 1; m < n; ++m)
        for (int p = 0; p <= n; ++p) {
            long double a = (p >= 1) ? (2 * m + 1) * P[m][p - 1] : 0.0L;
            P[m + 1][p] = (a - m * P[m - 1][p]) / (m + 1);
        }
    std::vector<long double> c = P[n];
    long double s = std::sqrt((2.0L * n + 1.0L) / 2.0L);
    for (auto& x : c) x *= s;
    return c;
}

static std::vector<std::array<int, 3>> basis_exponents(int D, int k) {
    std::vector<std::array<int, 3>> r;
    for (int deg = 0; deg <= k; ++deg) {
        if (D == 1) {
            r.push_back({deg, 0, 0});
        } else if (D == 2) {
            for (int ex = 0; ex <= deg; ++ex) r.push_back({ex, deg - ex, 0});
        } else {
            for (int ex = 0; ex <= deg; ++ex)
                for (int ey = 0; ey <= deg - ex; ++ey) r.push_back({ex, ey, deg - ex - ey});
        }
    }
    return r;
}

static std::vector<Poly> make_basis(int D, int k) {
    std::vector<Poly> B;
    std::vector<std::vector<long double>> L;
    for (int n = 0; n <= k; ++n) L.push_back(legendre_monomials(n));
    for (auto e : basis_exponents(D, k)) {
        Poly p;
        for (int a = 0; a <= e[0]; ++a)
            for (int b = 0; b <= (D >= 2 ? e[1] : 0); ++b)
                for (int c = 0; c <= (D >= 3 ? e[2] : 0); ++c) {
                    long double v = L[e[0]][a] * (D >= 2 ? L[e[1]][b] : 1.0L) * (D >= 3 ? L[e[2]][c] : 1.0L);
                    if (D == 1) v = L[e[0]][a];
                    if (v != 0.0L) {
                        p.coef.push_back((double)v);
                        p.exps.push_back({a, b, c});
                    }
                }
        B.push_back(p);
    }
    return B;
}

static double ipow(double x, int p) {
    double r = 1.0;
    for (int i = 0; i < p; ++i) r *= x;
    return r;
}

// value and reference-coordinate gradient of a polynomial at xi
static void poly_eval(const Poly& p, int D, const double* xi, double& val, double* grad) {
    val = 0;
    for (int d = 0; d < D; ++d) grad[d] = 0;
    for (size_t t = 0; t < p.coef.size(); ++t) {
        const auto& e = p.exps[t];
        double m[3], dm[3];
        for (int d = 0; d < D; ++d) {
            m[d] = ipow(xi[d], e[d]);
            dm[d] = e[d] > 0 ? e[d] * ipow(xi[d], e[d] - 1) : 0.0;
        }
        double prod = 1.0;
        for (int d = 0; d < D; ++d) prod *= m[d];
        val += p.coef[t] * prod;
        for (int d = 0; d < D; ++d) {
            double g = dm[d];
            for (int d2 = 0; d2 < D; ++d2)
                if (d2 != d) g *= m[d2];
            grad[d] += p.coef[t] * g;
        }
    }
}

// ------------------------------------------------------------------ Gauss rules
// Gauss-Legendre with n nodes (order 2n-1), ascending nodes, as in LineQuadRules.
static void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    const long double PI = 3.141592653589793238462643383279502884L;
    for (int i = 0; i < n; ++i) {
        long double z = std::cos(PI * (i + 0.75L) / (n + 0.5L));
        long double pp = 0;
        for (int it = 0; it < 100; ++it) {
            long double p0 = 1.0L, p1 = z;
            if (n == 0) break;
            for (int m = 1; m < n; ++m) {
                long double p2 = ((2 * m + 1) * z * p1 - m * p0) / (m + 1);
                p0 = p1;
                p1 = p2;
            }
            long double pn = (n == 1) ? z : p1;
            long double pnm1 = (n == 1) ? 1.0L : p0;
            pp = n * (z * pn - pnm1) / (z * z - 1.0L);
            long double dz = pn / pp;
            z -= dz;
            if (std::fabs((double)dz) < 1e-19) break;
        }
        {
            long double p0 = 1.0L, p1 = z;
            for (int m = 1; m < n; ++m) {
                long double p2 = ((2 * m + 1) * z * p1 - m * p0) / (m + 1);
                p0 = p1;
                p1 = p2;
            }
            long double pn = (n == 1) ? z : p1;
            long double pnm1 = (n == 1) ? 1.0L : p0;
            pp = n * (z * pn - pnm1) / (z * z - 1.0L);
        }
        x[n - 1 - i] = (double)z;
        w[n - 1 - i] = (double)(2.0L / ((1.0L - z * z) * pp * pp));
    }
    if (n % 2 == 1) x[n / 2] = 0.0;
}

// Tensor rule with the reference node ordering:
//   Square.cs:110-127: node[i*N+j] = (x_j, y_i)
//   Cube.cs:176-183:   node[(i*N+j)*N+k] = (x_k, y_j, z_i)
static void tensor_rule(int D, int n, std::vector<double>& nodes, std::vector<double>& wts) {
    std::vector<double> x, w;
    gauss_legendre(n, x, w);
    nodes.clear();
    wts.clear();
    if (D == 1) {
        for (int i = 0; i < n; ++i) { nodes.push_back(x[i]); wts.push_back(w[i]); }
    } else if (D == 2) {
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                nodes.push_back(x[j]);
                nodes.push_back(x[i]);
                wts.push_back(w[i] * w[j]);
            }
    } else {
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j)
                for (int k = 0; k < n; ++k) {
                    nodes.push_back(x[k]);
                    nodes.push_back(x[j]);
                    nodes.push_back(x[i]);
                    wts.push_back(w[i] * w[j] * w[k]);
                }
    }
}

// QuadOrderFunc.cs restated
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
            if (o % 2) ++o;
            return o;
        }
    }
    return -1;
}

// ------------------------------------------------------------------ problem
struct Problem {
    bosss_op_desc op;
    bosss_grid_desc g;
    int D;
    int J;                       // cells
    int nQ1;                     // Gauss nodes per direction
    std::vector<int> dom_np, dom_off, cod_np, cod_off;
    int dom_per_cell, cod_per_cell;
    double h[3], detJ, scaling, faceSG[3];
    std::vector<double> cj;      // 1 / CellLengthScale
    int pmax;                    // max domain degree (SIP penalty)
    // volume rule and tabulated basis (per degree)
    std::vector<double> vn, vw;  // nodes [Q][D], weights
    int maxdeg;
    std::vector<std::vector<Poly>> basis;   // per degree k: polys
    // volume tables per degree: phi[k][q*Np+n], dphi[k][(q*Np+n)*D+d]
    std::vector<std::vector<double>> vphi, vdphi;
    // face rule (D-1 dims)
    std::vector<double> fn, fw;
    int nQf;
    // face tables per degree (BasisData caches values at face nodes per face index):
    // fphi[k][((2d+s)*Qf + q)*Np + n], fdphi[k][(((2d+s)*Qf + q)*Np + n)*D + dd], s = 0 lower / 1 upper face
    std::vector<std::vector<double>> fphi, fdphi;
    // boundary-state table (nullable): outer values of every domain variable at every boundary
    // face node, bnd[node * n_domain + f]. Nodes are numbered cell by cell (storage order), then
    // face direction d, then side s (0 lower, 1 upper), then face node q; bnd_off[j*2D + 2d + s]
    // is the first node of that boundary face (-1: interior face).
    const double* bnd = nullptr;
    // boundary-condition kind per boundary face node (null: all 0): 0 the table's state, 1 the
    // inner state (SupersonicOutlet), 2 the inner state with the normal momentum reflected
    // (AdiabaticSlipWall); kinds 1 and 2 for the HLLC fluxes
    const int* kinds = nullptr;
    std::vector<long long> bnd_off;
    long long n_bnd_nodes = 0;
};

static int np_of(int D, int k) {
    if (k < 0) return 0;
    if (D == 1) return k + 1;
    if (D == 2) return (k + 1) * (k + 2) / 2;
    return (k + 1) * (k + 2) * (k + 3) / 6;
}

// 2D GlobalIDs (Grid2D.cs:182: ix*nY + iy) coincide with the generator order
static void cell_ijk(const Problem& P, int j, int* ijk) {
    const int* n = P.g.n;
    if (P.g.cell_order == BOSSS_CELLS_GENERATOR || P.D == 2) {
        if (P.D == 2) { ijk[0] = j / n[1]; ijk[1] = j % n[1]; ijk[2] = 0; }
        else { ijk[2] = j % n[2]; int r = j / n[2]; ijk[1] = r % n[1]; ijk[0] = r / n[1]; }
    } else {
        ijk[0] = j % n[0];
        int r = j / n[0];
        ijk[1] = r % n[1];
        ijk[2] = r / n[1];
    }
}

static int cell_index(const Problem& P, const int* ijk) {
    const int* n = P.g.n;
    if (P.g.cell_order == BOSSS_CELLS_GENERATOR || P.D == 2) {
        if (P.D == 2) return ijk[0] * n[1] + ijk[1];
        return (ijk[0] * n[1] + ijk[1]) * n[2] + ijk[2];
    }
    return ijk[0] + n[0] * (ijk[1] + n[1] * ijk[2]);
}

// neighbour across face (d, side): side 0 = lower, 1 = upper; -1 = boundary
static int neighbour(const Problem& P, int j, int d, int side) {
    int ijk[3];
    cell_ijk(P, j, ijk);
    ijk[d] += side ? 1 : -1;
    if (ijk[d] < 0 || ijk[d] >= P.g.n[d]) {
        if (!P.g.periodic[d]) return -1;
        ijk[d] = (ijk[d] + P.g.n[d]) % P.g.n[d];
    }
    return cell_index(P, ijk);
}

static int cell_index_along(const Problem& P, int j, int d) {
    int ijk[3];
    cell_ijk(P, j, ijk);
    return ijk[d];
}

static void cell_center(const Problem& P, int j, double* c) {
    int ijk[3];
    cell_ijk(P, j, ijk);
    for (int d = 0; d < P.D; ++d) c[d] = P.g.lo[d] + (ijk[d] + P.g.global_offset[d] + 0.5) * P.h[d];
}

static std::string setup(Problem& P, const bosss_op_desc* op, const bosss_grid_desc* g) {
    P.op = *op;
    P.g = *g;
    P.D = g->dim;
    if (P.D < 2 || P.D > 3) return "dim must be 2 or 3";
    P.J = 1;
    for (int d = 0; d < P.D; ++d) {
        if (g->n[d] < 1) return "bad n";
        P.J *= g->n[d];
        // a part's box is the global box (bosss_grid_desc): the cell width is the global one
        P.h[d] = (g->hi[d] - g->lo[d]) / (g->global_n[d] ? g->global_n[d] : g->n[d]);
    }
    P.detJ = 1;
    for (int d = 0; d < P.D; ++d) P.detJ *= 0.5 * P.h[d];
    P.scaling = 1.0 / std::sqrt(P.detJ);
    for (int d = 0; d < P.D; ++d) {
        double sg = 1;
        for (int d2 = 0; d2 < P.D; ++d2)
            if (d2 != d) sg *= 0.5 * P.h[d2];
        P.faceSG[d] = sg;
    }
    int o = quad_order(*op);
    if (o < 0) return "bad quad order";
    P.nQ1 = std::max(1, (o + 2) / 2);  // smallest n with 2n-1 >= o
    P.dom_np.clear(); P.dom_off.clear(); P.cod_np.clear(); P.cod_off.clear();
    int off = 0;
    P.maxdeg = 0;
    P.pmax = 0;
    for (int i = 0; i < op->n_domain; ++i) {
        P.dom_np.push_back(np_of(P.D, op->domain_degree[i]));
        P.dom_off.push_back(off);
        off += P.dom_np.back();
        P.maxdeg = std::max(P.maxdeg, op->domain_degree[i]);
        P.pmax = std::max(P.pmax, op->domain_degree[i]);
    }
    P.dom_per_cell = off;
    off = 0;
    for (int i = 0; i < op->n_codomain; ++i) {
        P.cod_np.push_back(np_of(P.D, op->codomain_degree[i]));
        P.cod_off.push_back(off);
        off += P.cod_np.back();
        P.maxdeg = std::max(P.maxdeg, op->codomain_degree[i]);
    }
    P.cod_per_cell = off;
    tensor_rule(P.D, P.nQ1, P.vn, P.vw);
    tensor_rule(P.D - 1, P.nQ1, P.fn, P.fw);
    P.nQf = (int)P.fw.size();
    P.basis.clear();
    P.vphi.clear();
    P.vdphi.clear();
    int Q = (int)P.vw.size();
    for (int k = 0; k <= P.maxdeg; ++k) {
        P.basis.push_back(make_basis(P.D, k));
        int Np = np_of(P.D, k);
        std::vector<double> phi(Q * Np), dphi(Q * Np * P.D);
        for (int q = 0; q < Q; ++q)
            for (int n = 0; n < Np; ++n) {
                double v, gr[3];
                poly_eval(P.basis[k][n], P.D, &P.vn[q * P.D], v, gr);
                phi[q * Np + n] = v;
                for (int d = 0; d < P.D; ++d) dphi[(q * Np + n) * P.D + d] = gr[d];
            }
        P.vphi.push_back(phi);
        P.vdphi.push_back(dphi);
    }
    P.fphi.clear();
    P.fdphi.clear();
    for (int k = 0; k <= P.maxdeg; ++k) {
        int Np = np_of(P.D, k), Qf = P.nQf;
        std::vector<double> phi((size_t)2 * P.D * Qf * Np), dphi((size_t)2 * P.D * Qf * Np * P.D);
        for (int d = 0; d < P.D; ++d)
            for (int s = 0; s < 2; ++s)
                for (int q = 0; q < Qf; ++q) {
                    double xi[3];
                    xi[d] = s ? 1.0 : -1.0;
                    int t = 0;
                    for (int d2 = 0; d2 < P.D; ++d2)
                        if (d2 != d) xi[d2] = P.fn[q * (P.D - 1) + t++];
                    for (int n = 0; n < Np; ++n) {
                        double v, gr[3];
                        poly_eval(P.basis[k][n], P.D, xi, v, gr);
                        size_t idx = ((size_t)(2 * d + s) * Qf + q) * Np + n;
                        phi[idx] = v;
                        for (int dd = 0; dd < P.D; ++dd) dphi[idx * P.D + dd] = gr[dd];
                    }
                }
        P.fphi.push_back(phi);
        P.fdphi.push_back(dphi);
    }
    // cj = (CellSurfaceArea + bndArea) * 0.5 / volume   (GridData_CellData.cs:663-684)
    bool part = false;
    for (int d = 0; d < P.D; ++d) part = part || g->global_n[d] != 0;
    P.cj.assign(P.J, 0.0);
    double vol = 1;
    for (int d = 0; d < P.D; ++d) vol *= P.h[d];
    for (int j = 0; j < P.J; ++j) {
        double surf = 0, bnd = 0;
        for (int d = 0; d < P.D; ++d) {
            double area = 1;
            for (int d2 = 0; d2 < P.D; ++d2)
                if (d2 != d) area *= P.h[d2];
            for (int s = 0; s < 2; ++s) {
                surf += area;
                bool boundary = neighbour(P, j, d, s) < 0;
                if (part) {
                    // part of a partitioned grid: only the global boundary counts
                    const int gi = cell_index_along(P, j, d) + g->global_offset[d];
                    boundary = !g->global_periodic[d] && (s == 0 ? gi == 0 : gi == g->global_n[d] - 1);
                }
                if (boundary) bnd += area;
            }
        }
        P.cj[j] = (surf + bnd) * 0.5 / vol;
    }
    // boundary face node numbering of the boundary-state table: faces on the boundary of the
    // (global) grid; the outer faces of a part's ghost planes have no table entry
    P.bnd_off.assign((size_t)P.J * 2 * P.D, -1);
    P.n_bnd_nodes = 0;
    for (int j = 0; j < P.J; ++j)
        for (int d = 0; d < P.D; ++d)
            for (int s = 0; s < 2; ++s) {
                bool boundary = neighbour(P, j, d, s) < 0;
                if (part) {
                    const int gi = cell_index_along(P, j, d) + g->global_offset[d];
                    boundary = !g->global_periodic[d] && (s == 0 ? gi == 0 : gi == g->global_n[d] - 1);
                }
                if (boundary) {
                    P.bnd_off[(size_t)j * 2 * P.D + 2 * d + s] = P.n_bnd_nodes;
                    P.n_bnd_nodes += P.nQf;
                }
            }
    // component checks
    for (int c = 0; c < op->n_components; ++c) {
        const auto& cp = op->components[c];
        if (cp.codomain < 0 || cp.codomain >= op->n_codomain) return "bad codomain index";
        for (int a = 0; a < cp.n_args; ++a)
            if (cp.args[a] < 0 || cp.args[a] >= op->n_domain) return "bad argument index";
        switch (cp.type) {
            case BOSSS_COMP_SCALAR_TRANSPORT_FLUX:
            case BOSSS_COMP_SIP_LAPLACE:
                if (cp.n_args != 1) return "component needs one argument";
                break;
            case BOSSS_COMP_CONSTANT_SOURCE: break;
            case BOSSS_COMP_HLLC_DENSITY_FLUX:
            case BOSSS_COMP_HLLC_MOMENTUM_FLUX:
            case BOSSS_COMP_HLLC_ENERGY_FLUX:
                if (cp.n_args != P.D + 2) return "HLLC needs D+2 arguments";
                break;
            case ORC_COMP_CNS_SIPG_DENSITY:
            case ORC_COMP_CNS_SIPG_MOMENTUM:
            case ORC_COMP_CNS_SIPG_ENERGY:
                if (cp.n_args != P.D + 2) return "CNS SIPG needs D+2 arguments";
                if (cp.type == ORC_COMP_CNS_SIPG_MOMENTUM && (cp.params[8] < 0 || cp.params[8] >= P.D))
                    return "CNS SIPG momentum: bad component";
                break;
            default: return "unsupported component";
        }
    }
    return "";
}

// ------------------------------------------------------------------ CNS viscous terms
// Hartmann's G tensor of the viscous flux of one conservation equation, F_k = sum_{l,j}
// G[k][l][j] dU_j/dx_l, as OptimizedSIPG{Momentum,Energy}Flux.UpdateTensorComponent and
// UpdateBoundaryTensorComponent set it (CNS/Diffusion/OptimizedSIPGMomentumFlux.cs:592-1000,
// OptimizedSIPGEnergyFlux.cs:630-956). U = conservative state (rho, m_0..m_{D-1}, rhoE).
// Velocity v = m / rho, temperature T = (gamma-1) (rhoE/rho - MachScaling |v|^2 / 2),
// mu_hat = mu(T) / (Re rho), MachScaling = gamma Mach^2, alpha = bulk viscosity ratio.
// Momentum equation c: the coefficients of tau_ck = mu (d_k v_c + d_c v_k) + (alpha - 2/3) mu
// delta_ck div v written on the conservative gradients (d_l v_i = (d_l m_i - v_i d_l rho)/rho).
// In two dimensions the y-momentum entry G[x][y][rho] of the reference is -v_y mu_hat (where
// the formula gives -v_x mu_hat); that entry is kept as the reference has it
// (OptimizedSIPGMomentumFlux.cs:767 and the boundary variant, SIPGMomentumFlux.cs:63).
// Energy equation: the reference's entries, in closed form (k flux direction, l gradient):
//   G[k][k][rho] = -(MS (alpha+1/3) v_k^2 + MS |v|^2 + gPr (e - MS |v|^2)) mu_hat
//   G[k][k][m_i] = MS (alpha+4/3 - gPr) v_k mu_hat (i = k),  MS (1 - gPr) v_i mu_hat (i != k)
//   G[k][k][rhoE] = gPr mu_hat,  gPr = gamma / Pr
//   G[k][l][rho] = -MS (alpha+1/3) v_k v_l mu_hat, G[k][l][m_k] = MS v_l mu_hat,
//   G[k][l][m_l] = MS (alpha-2/3) v_k mu_hat                                   (l != k)
template <class T>
static void cns_gtensor(const bosss_component& cp, int D, const T* U, T G[3][3][5]) {
    const double gamma = cp.params[0], Mach = cp.params[1], Re = cp.params[2], Pr = cp.params[3];
    const double alpha = cp.params[4];
    const double MS = gamma * Mach * Mach, gPr = gamma / Pr;
    const double a43 = alpha + 4.0 / 3.0, a23 = alpha - 2.0 / 3.0, a13 = alpha + 1.0 / 3.0;
    for (int k = 0; k < 3; ++k)
        for (int l = 0; l < 3; ++l)
            for (int j = 0; j < 5; ++j) G[k][l][j] = T(0.0);
    const T rho = U[cp.args[0]];
    T v[3];
    T q = T(0.0);
    for (int i = 0; i < D; ++i) {
        v[i] = U[cp.args[1 + i]] / rho;
        q += v[i] * v[i];
    }
    const T e = U[cp.args[D + 1]] / rho;
    const T temp = T(gamma - 1.0) * (e - T(0.5 * MS) * q);
    T mu = T(1.0);
    if (cp.params[5] == 1.0) {
        // SutherlandLaw.GetViscosity: T^{3/2} (1 + c) / (T + c)
        const double c = cp.params[6];
        mu = temp * sqrt(temp) * T(1.0 + c) / (temp + T(c));
    }
    const T mh = mu / T(Re) / rho;
    if (cp.type == ORC_COMP_CNS_SIPG_MOMENTUM) {
        const int c = (int)cp.params[8];
        for (int k = 0; k < D; ++k)
            for (int l = 0; l < D; ++l) {
                // coefficient of d_l v_i in tau_ck, for every i
                for (int i = 0; i < D; ++i) {
                    double coef = 0.0;
                    if (l == k && i == c) coef += 1.0;
                    if (l == c && i == k) coef += 1.0;
                    if (c == k && i == l) coef += a23;
                    if (coef == 0.0) continue;
                    G[k][l][0] -= T(coef) * v[i] * mh;
                    G[k][l][1 + i] += T(coef) * mh;
                }
            }
        if (D == 2 && c == 1) G[0][1][0] = -v[1] * mh;
    } else if (cp.type == ORC_COMP_CNS_SIPG_ENERGY) {
        for (int k = 0; k < D; ++k)
            for (int l = 0; l < D; ++l) {
                if (k == l) {
                    G[k][k][0] = -(T(MS) * (T(a13) * v[k] * v[k] + q) + T(gPr) * (e - T(MS) * q)) * mh;
                    for (int i = 0; i < D; ++i)
                        G[k][k][1 + i] = (i == k) ? T(MS * (a43 - gPr)) * v[k] * mh : T(MS * (1.0 - gPr)) * v[i] * mh;
                    G[k][k][D + 1] = T(gPr) * mh;
                } else {
                    G[k][l][0] = -T(MS * a13) * v[k] * v[l] * mh;
                    G[k][l][1 + k] = T(MS) * v[l] * mh;
                    G[k][l][1 + l] = T(MS * a23) * v[k] * mh;
                }
            }
    }
    // density: no viscous flux (OptimizedSIPGDensityFlux does nothing)
}

// SIPG penalty factor SIPGPenaltyScaling * p^2, p = the largest domain degree
// (OptimizedSIPGMomentumFlux.cs:118-119)
static double cns_penalty_factor(const Problem& P, const bosss_component& cp) {
    return cp.params[7] * (double)P.pmax * (double)P.pmax;
}

// ------------------------------------------------------------------ pointwise forms
// Volume: contributions fV (coefficient of v) and fG[d] (coefficient of grad v) for codomain var e.
template <class T>
static void volume_terms(const Problem& P, const bosss_component& cp, const T* U, const T (*G)[3],
                         const double* x, T& fV, T* fG) {
    const int D = P.D;
    switch (cp.type) {
        case BOSSS_COMP_SCALAR_TRANSPORT_FLUX: {
            // Flux = a*u; NECQuadratureVolume.cs:452 scales INonlinearFlux by -1
            T u = U[cp.args[0]];
            for (int d = 0; d < D; ++d) fG[d] -= cp.params[d] * u;
            break;
        }
        case BOSSS_COMP_SIP_LAPLACE: {
            // ipLaplace.cs VolumeForm: acc -= GradU[0,d]*GradV[d]*Nu
            T u = U[cp.args[0]];
            T nu = T(cp.params[1]) + T(cp.params[2]) * u * u;
            for (int d = 0; d < D; ++d) fG[d] -= G[cp.args[0]][d] * nu;
            break;
        }
        case BOSSS_COMP_CONSTANT_SOURCE: fV += T(cp.params[0]); break;
        case BOSSS_COMP_HLLC_DENSITY_FLUX: {
            // OptimizedHLLCDensityFlux.Flux: F_d = m_d, then scaled by -1
            for (int d = 0; d < D; ++d) fG[d] -= U[cp.args[1 + d]];
            break;
        }
        case BOSSS_COMP_HLLC_MOMENTUM_FLUX: {
            double gamma = cp.params[0], Mach = cp.params[1];
            int comp = (int)cp.params[2];
            double gMs = gamma * Mach * Mach;
            T rho = U[cp.args[0]], E = U[cp.args[D + 1]];
            T msq = T(0.0);
            T F[3];
            for (int d = 0; d < D; ++d) {
                F[d] = U[cp.args[comp + 1]] * U[cp.args[d + 1]] / rho;
                msq += U[cp.args[d + 1]] * U[cp.args[d + 1]];
            }
            T p = T(gamma - 1.0) * (E - T(gMs * 0.5) * msq / rho) / T(gMs);
            F[comp] += p;
            for (int d = 0; d < D; ++d) fG[d] -= F[d];
            break;
        }
        case BOSSS_COMP_HLLC_ENERGY_FLUX: {
            double gamma = cp.params[0], Mach = cp.params[1];
            double gMs = gamma * Mach * Mach;
            T rho = U[cp.args[0]], E = U[cp.args[D + 1]];
            T msq = T(0.0);
            for (int d = 0; d < D; ++d) msq += U[cp.args[d + 1]] * U[cp.args[d + 1]];
            T p = T(gamma - 1.0) * (E - T(gMs * 0.5) * msq / rho);
            for (int d = 0; d < D; ++d) fG[d] -= U[cp.args[d + 1]] / rho * (E + p);
            break;
        }
        case ORC_COMP_CNS_SIPG_DENSITY: break;
        case ORC_COMP_CNS_SIPG_MOMENTUM:
        case ORC_COMP_CNS_SIPG_ENERGY: {
            // INonlinVolumeForm_GradV.Form: f[k] += sum_{l,j} G[k][l][j] dU_j/dx_l
            T Gt[3][3][5];
            cns_gtensor(cp, D, U, Gt);
            for (int k = 0; k < D; ++k)
                for (int l = 0; l < D; ++l)
                    for (int j = 0; j < D + 2; ++j) fG[k] += Gt[k][l][j] * G[cp.args[j]][l];
            break;
        }
    }
}

// HLLC wave structure shared by the three OptimizedHLLC*Flux.InnerEdgeFlux methods.
template <class T>
struct HLLCState {
    T rhoIn, rhoOut, unIn, unOut, EIn, EOut, pIn, pOut, sIn, sOut, sStar;
};

template <class T>
static HLLCState<T> hllc_state(const T* Uin, const T* Uout, const int* args, int D, const double* n,
                               double gamma, double Mach) {
    HLLCState<T> s;
    double MachScaling = gamma * Mach * Mach;
    s.rhoIn = Uin[args[0]];
    s.rhoOut = Uout[args[0]];
    T msIn = T(0.0), msOut = T(0.0), unIn = T(0.0), unOut = T(0.0);
    for (int d = 0; d < D; ++d) {
        T mi = Uin[args[d + 1]], mo = Uout[args[d + 1]];
        msIn += mi * mi;
        msOut += mo * mo;
        unIn += mi * T(n[d]);
        unOut += mo * T(n[d]);
    }
    unIn /= s.rhoIn;
    unOut /= s.rhoOut;
    s.unIn = unIn;
    s.unOut = unOut;
    s.EIn = Uin[args[D + 1]];
    s.EOut = Uout[args[D + 1]];
    s.pIn = T(gamma - 1.0) * (s.EIn - T(MachScaling * 0.5) * msIn / s.rhoIn);
    s.pOut = T(gamma - 1.0) * (s.EOut - T(MachScaling * 0.5) * msOut / s.rhoOut);
    T cIn_snd = sqrt(s.pIn / s.rhoIn) / T(Mach);
    T cOut_snd = sqrt(s.pOut / s.rhoOut) / T(Mach);
    T rhoMean = T(0.5) * (s.rhoIn + s.rhoOut);
    T pMean = T(0.5) * (s.pIn + s.pOut);
    T cMean = T(0.5) * (cIn_snd + cOut_snd);
    T velJump = unOut - unIn;
    T pStar = pMean - T(0.5 * MachScaling) * velJump * cMean * rhoMean;
    pStar = tmax(T(0.0), pStar);
    T qIn = T(1.0), qOut = T(1.0);
    if (pStar > s.pIn) qIn = sqrt(T(1.0) + T(0.5 * (gamma + 1.0)) * (pStar / s.pIn - T(1.0)) / T(gamma));
    if (pStar > s.pOut) qOut = sqrt(T(1.0) + T(0.5 * (gamma + 1.0)) * (pStar / s.pOut - T(1.0)) / T(gamma));
    s.sIn = unIn - cIn_snd * qIn;
    s.sOut = unOut + cOut_snd * qOut;
    T cIn = s.rhoIn * (s.sIn - unIn);
    T cOut = s.rhoOut * (s.sOut - unOut);
    T speedDiff = cOut * unOut - cIn * unIn;
    T dp = s.pIn - s.pOut;
    s.sStar = (speedDiff + dp / T(MachScaling)) / (cOut - cIn);
    return s;
}

// Inner edge: returns (gA, GA[d], gB, GB[d]) = coefficients of vA, grad vA, vB, grad vB.
template <class T>
static void inner_edge_terms(const Problem& P, const bosss_component& cp, int jIn, int jOut, const T* UA,
                             const T (*GA)[3], const T* UB, const T (*GB)[3], const double* n,
                             T& gA, T* GAv, T& gB, T* GBv) {
    const int D = P.D;
    switch (cp.type) {
        case BOSSS_COMP_SCALAR_TRANSPORT_FLUX: {
            // TransportFlux.cs InnerEdgeFlux: upwind on the averaged velocity (constant here)
            T uin = UA[cp.args[0]], uout = UB[cp.args[0]];
            double an = 0;
            for (int d = 0; d < D; ++d) an += cp.params[d] * n[d];
            T f = (an > 0) ? T(an) * uin : T(an) * uout;
            gA += f;       // NECQuadratureEdge: IN +flux
            gB -= f;       // OUT = -IN (:998-1000)
            break;
        }
        case BOSSS_COMP_SIP_LAPLACE: {
            int a = cp.args[0];
            double pdeg = (P.pmax + 1.0) * (P.pmax + 1.0);
            double ptri = (P.pmax + 1.0) * (P.pmax + D) / D;
            double pen_deg = std::max(ptri, pdeg);
            double pnlty = std::max(cp.params[0] * pen_deg * P.cj[jIn], cp.params[0] * pen_deg * P.cj[jOut]);
            T uA = UA[a], uB = UB[a];
            T nuA = T(cp.params[1]) + T(cp.params[2]) * uA * uA;
            T nuB = T(cp.params[1]) + T(cp.params[2]) * uB * uB;
            T jump = uA - uB;
            for (int d = 0; d < D; ++d) {
                T cons = T(0.5) * (nuA * GA[a][d] + nuB * GB[a][d]) * T(n[d]);  // consistency
                gA += cons;
                gB -= cons;
                GAv[d] += T(0.5) * nuA * jump * T(n[d]);   // symmetry
                GBv[d] += T(0.5) * nuB * jump * T(n[d]);
            }
            T nuMax = (tabs(nuA) > tabs(nuB)) ? nuA : nuB;
            T pen = jump * T(pnlty) * nuMax;
            gA -= pen;
            gB += pen;
            break;
        }
        case ORC_COMP_CNS_SIPG_DENSITY: break;
        case ORC_COMP_CNS_SIPG_MOMENTUM:
        case ORC_COMP_CNS_SIPG_ENERGY: {
            // NonlinInternalEdge_V and _GradV (OptimizedSIPGMomentumFlux.cs:187-265, 343-449)
            const double pen = cns_penalty_factor(P, cp) * std::max(P.cj[jIn], P.cj[jOut]);
            T Gi[3][3][5], Go[3][3][5];
            cns_gtensor(cp, D, UA, Gi);
            cns_gtensor(cp, D, UB, Go);
            T flux = T(0.0);
            for (int k = 0; k < D; ++k) {
                T accIn = T(0.0), accOut = T(0.0);
                for (int l = 0; l < D; ++l)
                    for (int j = 0; j < D + 2; ++j) {
                        const int a = cp.args[j];
                        const T jump = UA[a] - UB[a];
                        flux -= T(0.5) * (Gi[k][l][j] * GA[a][l] + Go[k][l][j] * GB[a][l]) * T(n[k]);
                        flux += T(0.5) * (Gi[k][l][j] + Go[k][l][j]) * jump * T(n[l] * pen * n[k]);
                        accIn -= T(0.5) * Gi[k][l][j] * jump * T(n[l]);
                        accOut -= T(0.5) * Go[k][l][j] * jump * T(n[l]);
                    }
                GAv[k] += accIn;
                GBv[k] += accOut;
            }
            gA += flux;
            gB -= flux;
            break;
        }
        case BOSSS_COMP_CONSTANT_SOURCE: break;
        case BOSSS_COMP_HLLC_DENSITY_FLUX:
        case BOSSS_COMP_HLLC_MOMENTUM_FLUX:
        case BOSSS_COMP_HLLC_ENERGY_FLUX: {
            double gamma = cp.params[0], Mach = cp.params[1];
            double MachScaling = gamma * Mach * Mach;
            HLLCState<T> s = hllc_state(UA, UB, cp.args, D, n, gamma, Mach);
            T f = T(0.0);
            if (cp.type == BOSSS_COMP_HLLC_DENSITY_FLUX) {
                if (s.sStar > 0.0) {
                    f = s.unIn * s.rhoIn;
                    if (s.sIn <= 0.0) {
                        T mod = s.rhoIn * (s.sIn - s.unIn) / (s.sIn - s.sStar);
                        f += s.sIn * (mod - s.rhoIn);
                    }
                } else {
                    f = s.unOut * s.rhoOut;
                    if (s.sOut >= 0.0) {
                        T mod = s.rhoOut * (s.sOut - s.unOut) / (s.sOut - s.sStar);
                        f += s.sOut * (mod - s.rhoOut);
                    }
                }
            } else if (cp.type == BOSSS_COMP_HLLC_MOMENTUM_FLUX) {
                int c = (int)cp.params[2];
                T mIn = UA[cp.args[c + 1]], mOut = UB[cp.args[c + 1]];
                if (s.sStar > 0.0) {
                    f = s.unIn * mIn + s.pIn / T(MachScaling) * T(n[c]);
                    if (s.sIn <= 0.0) {
                        T mod = s.rhoIn * (s.sIn - s.unIn) / (s.sIn - s.sStar) *
                                (mIn / s.rhoIn + (s.sStar - s.unIn) * T(n[c]));
                        f += s.sIn * (mod - mIn);
                    }
                } else {
                    f = s.unOut * mOut + s.pOut / T(MachScaling) * T(n[c]);
                    if (s.sOut >= 0.0) {
                        T mod = s.rhoOut * (s.sOut - s.unOut) / (s.sOut - s.sStar) *
                                (mOut / s.rhoOut + (s.sStar - s.unOut) * T(n[c]));
                        f += s.sOut * (mod - mOut);
                    }
                }
            } else {
                if (s.sStar > 0.0) {
                    f = s.unIn * (s.EIn + s.pIn);
                    if (s.sIn <= 0.0) {
                        T factor = s.rhoIn * s.sStar * T(MachScaling) + s.pIn / (s.sIn - s.unIn);
                        T mod = (s.sIn - s.unIn) / (s.sIn - s.sStar) * (s.EIn + factor * (s.sStar - s.unIn));
                        f += s.sIn * (mod - s.EIn);
                    }
                } else {
                    f = s.unOut * (s.EOut + s.pOut);
                    if (s.sOut >= 0.0) {
                        T factor = s.rhoOut * s.sStar * T(MachScaling) + s.pOut / (s.sOut - s.unOut);
                        T mod = (s.sOut - s.unOut) / (s.sOut - s.sStar) * (s.EOut + factor * (s.sStar - s.unOut));
                        f += s.sOut * (mod - s.EOut);
                    }
                }
            }
            gA += f;
            gB -= f;
            break;
        }
    }
}

// Boundary edge (outward normal n): (gA, GA[d]).
// Ubnd: the boundary-state table's outer values of the domain variables at this node (null if
// the problem has no table).
template <class T>
static void boundary_edge_terms(const Problem& P, const bosss_component& cp, int jIn, const T* UA,
                                const T (*GA)[3], const double* n, const double* x, const double* Ubnd, int kind,
                                T& gA, T* GAv) {
    const int D = P.D;
    switch (cp.type) {
        case BOSSS_COMP_SCALAR_TRANSPORT_FLUX: {
            T uin = UA[cp.args[0]];
            double an = 0;
            for (int d = 0; d < D; ++d) an += cp.params[d] * n[d];
            if (D == 2) {
                gA += T(an) * uin;  // TransportFlux.cs:52-63: (vel*Uin)*n on in- and outflow
            } else {
                if (an >= 0) gA += T(an) * uin;  // TransportFlux.cs:143-151: inflow value 0
            }
            break;
        }
        case BOSSS_COMP_SIP_LAPLACE: {
            int a = cp.args[0];
            double pdeg = (P.pmax + 1.0) * (P.pmax + 1.0);
            double ptri = (P.pmax + 1.0) * (P.pmax + D) / D;
            double pen_deg = std::max(ptri, pdeg);
            double pnlty = 2.0 * cp.params[0] * pen_deg * P.cj[jIn];
            T uA = UA[a];
            T nuA = T(cp.params[1]) + T(cp.params[2]) * uA * uA;
            if (cp.params[3] == 0.0) {
                double gD = cp.params[4];
                for (int d = 0; d < D; ++d) gD += cp.params[5 + d] * x[d] + cp.params[8 + d] * x[d] * x[d];
                T diff = uA - T(gD);
                for (int d = 0; d < D; ++d) {
                    gA += nuA * GA[a][d] * T(n[d]);
                    GAv[d] += nuA * diff * T(n[d]);
                }
                gA -= nuA * diff * T(pnlty);
            }
            // Neumann with g_N = 0 contributes nothing
            break;
        }
        case ORC_COMP_CNS_SIPG_MOMENTUM:
        case ORC_COMP_CNS_SIPG_ENERGY: {
            // NonlinBoundaryEdge_V and _GradV (OptimizedSIPGMomentumFlux.cs:267-336, 451-540): the
            // G tensor of the outer state (SupersonicInlet.GetBoundaryState), penalty p^2 cj(in)
            if (!Ubnd) break;   // rejected by the entry points
            const double pen = cns_penalty_factor(P, cp) * P.cj[jIn];
            T Ub[BOSSS_MAX_VARS];
            for (int f = 0; f < P.op.n_domain; ++f) Ub[f] = T(Ubnd[f]);
            T Go[3][3][5];
            cns_gtensor(cp, D, Ub, Go);
            T flux = T(0.0);
            for (int k = 0; k < D; ++k)
                for (int l = 0; l < D; ++l)
                    for (int j = 0; j < D + 2; ++j) {
                        const int a = cp.args[j];
                        const T jump = UA[a] - Ub[a];
                        flux -= Go[k][l][j] * GA[a][l] * T(n[k]);
                        flux += Go[k][l][j] * jump * T(n[l] * pen * n[k]);
                        GAv[k] -= Go[k][l][j] * jump * T(n[l]);
                    }
            gA += flux;
            break;
        }
        case BOSSS_COMP_HLLC_DENSITY_FLUX:
        case BOSSS_COMP_HLLC_MOMENTUM_FLUX:
        case BOSSS_COMP_HLLC_ENERGY_FLUX: {
            // OptimizedHLLCFlux.BorderEdgeFlux (OptimizedHLLCFlux.cs:61-131): Uout from the
            // boundary condition, then InnerEdgeFlux(Uin, Uout) with the outward normal; only the
            // IN side is kept. Uout: the table's state (kind 0), Uin (SupersonicOutlet.cs, kind 1),
            // Uin with m - 2 (m . n) n (AdiabaticSlipWall.cs, kind 2)
            if (kind == 0 && !Ubnd) break;   // rejected by the entry points
            T Ub[BOSSS_MAX_VARS];
            T GB[BOSSS_MAX_VARS][3];
            T mn = T(0.0);
            for (int d = 0; d < D; ++d) mn += UA[cp.args[1 + d]] * T(n[d]);
            for (int f = 0; f < P.op.n_domain; ++f) {
                Ub[f] = (kind == 0) ? T(Ubnd[f]) : UA[f];
                for (int d = 0; d < 3; ++d) GB[f][d] = T(0.0);
            }
            if (kind == 2)
                for (int d = 0; d < D; ++d) Ub[cp.args[1 + d]] = UA[cp.args[1 + d]] - T(2.0) * mn * T(n[d]);
            T gB = T(0.0), GBv[3] = {T(0.0), T(0.0), T(0.0)};
            inner_edge_terms(P, cp, jIn, jIn, UA, GA, (const T*)Ub, (const T(*)[3])GB, n, gA, GAv, gB, GBv);
            (void)x;
            break;
        }
        default: break;
    }
}

// ------------------------------------------------------------------ evaluation
// outer values of the boundary-state table at node q of boundary face (j, d, s), or null
static const double* bnd_node(const Problem& P, int j, int d, int s, int q) {
    if (!P.bnd) return nullptr;
    const long long o = P.bnd_off[(size_t)j * 2 * P.D + 2 * d + s];
    return o < 0 ? nullptr : P.bnd + (size_t)(o + q) * P.op.n_domain;
}

// boundary-condition kind at node q of boundary face (j, d, s)
static int bnd_kind(const Problem& P, int j, int d, int s, int q) {
    if (!P.kinds) return 0;
    const long long o = P.bnd_off[(size_t)j * 2 * P.D + 2 * d + s];
    return o < 0 ? 0 : P.kinds[o + q];
}

// vflags / fflags (nullable): XDG species masks -- a cell's volume integral is taken only where
// vflags[j] == 1, a face only where fflags[j*2D + 2d + s] == 1 (interior faces by their lower
// cell's upper side, s = 1)
template <class T>
static void evaluate(const Problem& P, double alpha, double beta, const T* U, T* out,
                     const unsigned char* vflags = nullptr, const unsigned char* fflags = nullptr) {
    const int D = P.D, J = P.J, Q = (int)P.vw.size(), nd = P.op.n_domain, nc = P.op.n_codomain;
    const int Nd = P.dom_per_cell, Nc = P.cod_per_cell;
    // output *= beta  (DifferentialOperator.cs:1593-1594)
    for (long i = 0; i < (long)J * Nc; ++i) out[i] = T(beta) * out[i];

    // ---- volume (NECQuadratureVolume.EvaluateEx)
#pragma omp parallel for schedule(static)
    for (int j = 0; j < J; ++j) {
        if (vflags && vflags[j] != 1) continue;
        std::vector<T> R(Nc, T(0.0));
        double c[3];
        cell_center(P, j, c);
        for (int q = 0; q < Q; ++q) {
            T Uq[BOSSS_MAX_VARS], Gq[BOSSS_MAX_VARS][3];
            for (int f = 0; f < nd; ++f) {
                int k = P.op.domain_degree[f], Np = P.dom_np[f];
                T v = T(0.0), gr[3] = {T(0.0), T(0.0), T(0.0)};
                for (int n = 0; n < Np; ++n) {
                    T cf = U[(long)j * Nd + P.dom_off[f] + n];
                    v += cf * T(P.vphi[k][q * Np + n]);
                    for (int d = 0; d < D; ++d) gr[d] += cf * T(P.vdphi[k][(q * Np + n) * D + d]);
                }
                Uq[f] = v * T(P.scaling);
                for (int d = 0; d < D; ++d) Gq[f][d] = gr[d] * T(P.scaling * 2.0 / P.h[d]);
            }
            double x[3];
            for (int d = 0; d < D; ++d) x[d] = c[d] + 0.5 * P.h[d] * P.vn[q * D + d];
            for (int e = 0; e < nc; ++e) {
                T fV = T(0.0), fG[3] = {T(0.0), T(0.0), T(0.0)};
                for (int ci = 0; ci < P.op.n_components; ++ci)
                    if (P.op.components[ci].codomain == e)
                        volume_terms(P, P.op.components[ci], Uq, Gq, x, fV, fG);
                int k = P.op.codomain_degree[e], Np = P.cod_np[e];
                double w = P.vw[q];
                for (int m = 0; m < Np; ++m) {
                    T acc = fV * T(P.vphi[k][q * Np + m]);
                    for (int d = 0; d < D; ++d) acc += fG[d] * T(P.vdphi[k][(q * Np + m) * D + d] * 2.0 / P.h[d]);
                    R[P.cod_off[e] + m] += T(w) * acc;
                }
            }
        }
        for (int i = 0; i < Nc; ++i) out[(long)j * Nc + i] += T(alpha) * (R[i] * T(P.detJ * P.scaling));
    }

    // ---- edges (NECQuadratureEdge.EvaluateEx): list of (cellIn, cellOut or -1, direction, normal sign)
    struct Edge { int in, out, d; double sgn; };
    std::vector<Edge> edges;
    auto on = [&](int j, int d, int s) { return !fflags || fflags[(size_t)j * 2 * D + 2 * d + s] == 1; };
    for (int d = 0; d < D; ++d)
        for (int j = 0; j < J; ++j) {
            int up = neighbour(P, j, d, 1);
            if (on(j, d, 1)) edges.push_back({j, up >= 0 ? up : -1, d, 1.0});
            if (neighbour(P, j, d, 0) < 0 && on(j, d, 0)) edges.push_back({j, -1, d, -1.0});
        }
    const int E = (int)edges.size();
    std::vector<T> Rin((size_t)E * Nc, T(0.0)), Rout((size_t)E * Nc, T(0.0));
    const int Qf = P.nQf;
#pragma omp parallel for schedule(static)
    for (int ei = 0; ei < E; ++ei) {
        const Edge& ed = edges[ei];
        int d = ed.d;
        double nrm[3] = {0, 0, 0};
        nrm[d] = ed.sgn;
        int oth[2], no = 0;
        for (int d2 = 0; d2 < D; ++d2)
            if (d2 != d) oth[no++] = d2;
        double cIn[3], cOut[3];
        cell_center(P, ed.in, cIn);
        if (ed.out >= 0) cell_center(P, ed.out, cOut);
        for (int q = 0; q < Qf; ++q) {
            // face node in each cell's reference coordinates
            double xiIn[3], x[3];
            xiIn[d] = ed.sgn;
            for (int t = 0; t < D - 1; ++t) {
                xiIn[oth[t]] = P.fn[q * (D - 1) + t];
            }
            for (int d2 = 0; d2 < D; ++d2) x[d2] = cIn[d2] + 0.5 * P.h[d2] * xiIn[d2];
            T UA[BOSSS_MAX_VARS], GA[BOSSS_MAX_VARS][3], UB[BOSSS_MAX_VARS], GB[BOSSS_MAX_VARS][3];
            const int fIn = 2 * d + (ed.sgn > 0 ? 1 : 0), fOut = 2 * d + (ed.sgn > 0 ? 0 : 1);
            for (int side = 0; side < 2; ++side) {
                if (side == 1 && ed.out < 0) break;
                int jc = side ? ed.out : ed.in;
                int fi = side ? fOut : fIn;
                for (int f = 0; f < nd; ++f) {
                    int k = P.op.domain_degree[f], Np = P.dom_np[f];
                    const double* tp = &P.fphi[k][((size_t)fi * Qf + q) * Np];
                    const double* tg = &P.fdphi[k][((size_t)fi * Qf + q) * Np * D];
                    T v = T(0.0), gr[3] = {T(0.0), T(0.0), T(0.0)};
                    for (int n = 0; n < Np; ++n) {
                        T cf = U[(long)jc * Nd + P.dom_off[f] + n];
                        v += cf * T(tp[n]);
                        for (int dd = 0; dd < D; ++dd) gr[dd] += cf * T(tg[n * D + dd]);
                    }
                    T* Uo = side ? UB : UA;
                    T(*Go)[3] = side ? GB : GA;
                    Uo[f] = v * T(P.scaling);
                    for (int dd = 0; dd < D; ++dd) Go[f][dd] = gr[dd] * T(P.scaling * 2.0 / P.h[dd]);
                }
            }
            double wq = P.fw[q] * P.faceSG[d];
            for (int e = 0; e < nc; ++e) {
                T gA = T(0.0), gB = T(0.0), GAv[3] = {T(0.0), T(0.0), T(0.0)}, GBv[3] = {T(0.0), T(0.0), T(0.0)};
                for (int ci = 0; ci < P.op.n_components; ++ci) {
                    const auto& cp = P.op.components[ci];
                    if (cp.codomain != e) continue;
                    if (ed.out >= 0) inner_edge_terms(P, cp, ed.in, ed.out, UA, GA, UB, GB, nrm, gA, GAv, gB, GBv);
                    else boundary_edge_terms(P, cp, ed.in, UA, GA, nrm, x, bnd_node(P, ed.in, d, fIn % 2, q),
                                             bnd_kind(P, ed.in, d, fIn % 2, q), gA, GAv);
                }
                int k = P.op.codomain_degree[e], Np = P.cod_np[e];
                const double* ip = &P.fphi[k][((size_t)fIn * Qf + q) * Np];
                const double* ig = &P.fdphi[k][((size_t)fIn * Qf + q) * Np * D];
                const double* op_ = &P.fphi[k][((size_t)fOut * Qf + q) * Np];
                const double* og = &P.fdphi[k][((size_t)fOut * Qf + q) * Np * D];
                for (int m = 0; m < Np; ++m) {
                    T acc = gA * T(ip[m]);
                    for (int dd = 0; dd < D; ++dd) acc += GAv[dd] * T(ig[m * D + dd] * 2.0 / P.h[dd]);
                    Rin[(size_t)ei * Nc + P.cod_off[e] + m] += T(wq * P.scaling) * acc;
                    if (ed.out >= 0) {
                        T acc2 = gB * T(op_[m]);
                        for (int dd = 0; dd < D; ++dd) acc2 += GBv[dd] * T(og[m * D + dd] * 2.0 / P.h[dd]);
                        Rout[(size_t)ei * Nc + P.cod_off[e] + m] += T(wq * P.scaling) * acc2;
                    }
                }
            }
        }
    }
    // scatter (SaveIntegrationResults): serial, in edge order
    for (int ei = 0; ei < E; ++ei) {
        const Edge& ed = edges[ei];
        for (int i = 0; i < Nc; ++i) out[(long)ed.in * Nc + i] += T(alpha) * Rin[(size_t)ei * Nc + i];
        if (ed.out >= 0)
            for (int i = 0; i < Nc; ++i) out[(long)ed.out * Nc + i] += T(alpha) * Rout[(size_t)ei * Nc + i];
    }
}

// ------------------------------------------------------------------ adjoint product
// out = J(U)^T W: the gradient of Phi(U) = W . Op(U) (alpha = 1, beta = 0). Volume node q of
// cell j contributes w_q detJ Scaling sum_e (fV_e lam_e + fG_e . grad lam_e), lam_e = W of
// codomain field e interpolated with its test functions; an edge node contributes the same
// with both cells' test functions (IN and OUT sides as in the evaluation). Each contribution
// is differentiated with respect to the node states (values and gradients of the domain
// fields) of the cells it reads, with N dual slots (own cell first, then the OUT cell), and
// the node-state derivatives are chained to the coefficients through the basis tables.
template <int N>
static void vjp(const Problem& P, const double* U, const double* W, double* out) {
    using T = DualV<N>;
    const int D = P.D, J = P.J, Q = (int)P.vw.size(), nd = P.op.n_domain, nc = P.op.n_codomain;
    const int Nd = P.dom_per_cell, Nc = P.cod_per_cell, S1 = nd * (1 + D);
    for (long i = 0; i < (long)J * Nd; ++i) out[i] = 0.0;

    // ---- volume (each cell writes its own entries)
#pragma omp parallel for schedule(static)
    for (int j = 0; j < J; ++j) {
        double c[3];
        cell_center(P, j, c);
        for (int q = 0; q < Q; ++q) {
            T Uq[BOSSS_MAX_VARS], Gq[BOSSS_MAX_VARS][3];
            for (int f = 0; f < nd; ++f) {
                int k = P.op.domain_degree[f], Np = P.dom_np[f];
                double v = 0, gr[3] = {0, 0, 0};
                for (int n = 0; n < Np; ++n) {
                    double cf = U[(long)j * Nd + P.dom_off[f] + n];
                    v += cf * P.vphi[k][q * Np + n];
                    for (int d = 0; d < D; ++d) gr[d] += cf * P.vdphi[k][(q * Np + n) * D + d];
                }
                Uq[f] = T(v * P.scaling);
                Uq[f].d[f * (1 + D)] = 1.0;
                for (int d = 0; d < D; ++d) {
                    Gq[f][d] = T(gr[d] * P.scaling * 2.0 / P.h[d]);
                    Gq[f][d].d[f * (1 + D) + 1 + d] = 1.0;
                }
            }
            double x[3];
            for (int d = 0; d < D; ++d) x[d] = c[d] + 0.5 * P.h[d] * P.vn[q * D + d];
            T phi = T(0.0);
            for (int e = 0; e < nc; ++e) {
                T fV = T(0.0), fG[3] = {T(0.0), T(0.0), T(0.0)};
                for (int ci = 0; ci < P.op.n_components; ++ci)
                    if (P.op.components[ci].codomain == e) volume_terms(P, P.op.components[ci], Uq, Gq, x, fV, fG);
                int k = P.op.codomain_degree[e], Np = P.cod_np[e];
                double lam = 0, glam[3] = {0, 0, 0};
                for (int m = 0; m < Np; ++m) {
                    const double wv = W[(long)j * Nc + P.cod_off[e] + m];
                    lam += wv * P.vphi[k][q * Np + m];
                    for (int d = 0; d < D; ++d) glam[d] += wv * P.vdphi[k][(q * Np + m) * D + d] * 2.0 / P.h[d];
                }
                phi += fV * T(lam);
                for (int d = 0; d < D; ++d) phi += fG[d] * T(glam[d]);
            }
            const double wq = P.vw[q] * P.detJ * P.scaling;
            for (int f = 0; f < nd; ++f) {
                int k = P.op.domain_degree[f], Np = P.dom_np[f];
                for (int n = 0; n < Np; ++n) {
                    double acc = phi.d[f * (1 + D)] * P.vphi[k][q * Np + n];
                    for (int d = 0; d < D; ++d)
                        acc += phi.d[f * (1 + D) + 1 + d] * P.vdphi[k][(q * Np + n) * D + d] * 2.0 / P.h[d];
                    out[(long)j * Nd + P.dom_off[f] + n] += wq * P.scaling * acc;
                }
            }
        }
    }

    // ---- edges: per-edge contributions to both cells, scattered afterwards
    struct Edge { int in, out, d; double sgn; };
    std::vector<Edge> edges;
    for (int d = 0; d < D; ++d)
        for (int j = 0; j < J; ++j) {
            int up = neighbour(P, j, d, 1);
            edges.push_back({j, up >= 0 ? up : -1, d, 1.0});
            if (neighbour(P, j, d, 0) < 0) edges.push_back({j, -1, d, -1.0});
        }
    const int E = (int)edges.size(), Qf = P.nQf;
    std::vector<double> Gin((size_t)E * Nd, 0.0), Gout((size_t)E * Nd, 0.0);
#pragma omp parallel for schedule(static)
    for (int ei = 0; ei < E; ++ei) {
        const Edge& ed = edges[ei];
        const int d = ed.d;
        double nrm[3] = {0, 0, 0};
        nrm[d] = ed.sgn;
        int oth[2], no = 0;
        for (int d2 = 0; d2 < D; ++d2)
            if (d2 != d) oth[no++] = d2;
        double cIn[3];
        cell_center(P, ed.in, cIn);
        const int fIn = 2 * d + (ed.sgn > 0 ? 1 : 0), fOut = 2 * d + (ed.sgn > 0 ? 0 : 1);
        for (int q = 0; q < Qf; ++q) {
            double xiIn[3], x[3];
            xiIn[d] = ed.sgn;
            for (int t = 0; t < D - 1; ++t) xiIn[oth[t]] = P.fn[q * (D - 1) + t];
            for (int d2 = 0; d2 < D; ++d2) x[d2] = cIn[d2] + 0.5 * P.h[d2] * xiIn[d2];
            T UA[BOSSS_MAX_VARS], GA[BOSSS_MAX_VARS][3], UB[BOSSS_MAX_VARS], GB[BOSSS_MAX_VARS][3];
            for (int side = 0; side < 2; ++side) {
                if (side == 1 && ed.out < 0) break;
                const int jc = side ? ed.out : ed.in, fi = side ? fOut : fIn, s0 = side * S1;
                for (int f = 0; f < nd; ++f) {
                    int k = P.op.domain_degree[f], Np = P.dom_np[f];
                    const double* tp = &P.fphi[k][((size_t)fi * Qf + q) * Np];
                    const double* tg = &P.fdphi[k][((size_t)fi * Qf + q) * Np * D];
                    double v = 0, gr[3] = {0, 0, 0};
                    for (int n = 0; n < Np; ++n) {
                        double cf = U[(long)jc * Nd + P.dom_off[f] + n];
                        v += cf * tp[n];
                        for (int dd = 0; dd < D; ++dd) gr[dd] += cf * tg[n * D + dd];
                    }
                    T* Uo = side ? UB : UA;
                    T(*Go)[3] = side ? GB : GA;
                    Uo[f] = T(v * P.scaling);
                    Uo[f].d[s0 + f * (1 + D)] = 1.0;
                    for (int dd = 0; dd < D; ++dd) {
                        Go[f][dd] = T(gr[dd] * P.scaling * 2.0 / P.h[dd]);
                        Go[f][dd].d[s0 + f * (1 + D) + 1 + dd] = 1.0;
                    }
                }
            }
            T phi = T(0.0);
            for (int e = 0; e < nc; ++e) {
                T gA = T(0.0), gB = T(0.0), GAv[3] = {T(0.0), T(0.0), T(0.0)}, GBv[3] = {T(0.0), T(0.0), T(0.0)};
                for (int ci = 0; ci < P.op.n_components; ++ci) {
                    const auto& cp = P.op.components[ci];
                    if (cp.codomain != e) continue;
                    if (ed.out >= 0) inner_edge_terms(P, cp, ed.in, ed.out, UA, GA, UB, GB, nrm, gA, GAv, gB, GBv);
                    else boundary_edge_terms(P, cp, ed.in, UA, GA, nrm, x, bnd_node(P, ed.in, d, fIn % 2, q),
                                             bnd_kind(P, ed.in, d, fIn % 2, q), gA, GAv);
                }
                int k = P.op.codomain_degree[e], Np = P.cod_np[e];
                for (int side = 0; side < 2; ++side) {
                    if (side == 1 && ed.out < 0) break;
                    const int jc = side ? ed.out : ed.in, fi = side ? fOut : fIn;
                    const double* tp = &P.fphi[k][((size_t)fi * Qf + q) * Np];
                    const double* tg = &P.fdphi[k][((size_t)fi * Qf + q) * Np * D];
                    double lam = 0, glam[3] = {0, 0, 0};
                    for (int m = 0; m < Np; ++m) {
                        const double wv = W[(long)jc * Nc + P.cod_off[e] + m];
                        lam += wv * tp[m];
                        for (int dd = 0; dd < D; ++dd) glam[dd] += wv * tg[m * D + dd] * 2.0 / P.h[dd];
                    }
                    phi += (side ? gB : gA) * T(lam);
                    for (int dd = 0; dd < D; ++dd) phi += (side ? GBv[dd] : GAv[dd]) * T(glam[dd]);
                }
            }
            const double wq = P.fw[q] * P.faceSG[d] * P.scaling;
            for (int side = 0; side < 2; ++side) {
                if (side == 1 && ed.out < 0) break;
                const int fi = side ? fOut : fIn, s0 = side * S1;
                double* Gb = side ? &Gout[(size_t)ei * Nd] : &Gin[(size_t)ei * Nd];
                for (int f = 0; f < nd; ++f) {
                    int k = P.op.domain_degree[f], Np = P.dom_np[f];
                    const double* tp = &P.fphi[k][((size_t)fi * Qf + q) * Np];
                    const double* tg = &P.fdphi[k][((size_t)fi * Qf + q) * Np * D];
                    for (int n = 0; n < Np; ++n) {
                        double acc = phi.d[s0 + f * (1 + D)] * tp[n];
                        for (int dd = 0; dd < D; ++dd)
                            acc += phi.d[s0 + f * (1 + D) + 1 + dd] * tg[n * D + dd] * 2.0 / P.h[dd];
                        Gb[P.dom_off[f] + n] += wq * P.scaling * acc;
                    }
                }
            }
        }
    }
    for (int ei = 0; ei < E; ++ei) {
        const Edge& ed = edges[ei];
        for (int i = 0; i < Nd; ++i) out[(long)ed.in * Nd + i] += Gin[(size_t)ei * Nd + i];
        if (ed.out >= 0)
            for (int i = 0; i < Nd; ++i) out[(long)ed.out * Nd + i] += Gout[(size_t)ei * Nd + i];
    }
}

static thread_local std::string g_err;

// ------------------------------------------------------------------ XDG bulk (given rules)
// Volume integral of cell j with reference nodes xi[npts*D] and weights w[npts]
// (NECQuadratureVolume semantics with a cut-cell rule), added to R[Nc].
static void vol_integral(const Problem& P, int j, int npts, const double* xi, const double* w, const double* U,
                         double* R) {
    const int D = P.D, nd = P.op.n_domain, nc = P.op.n_codomain, Nd = P.dom_per_cell;
    double c[3];
    cell_center(P, j, c);
    for (int q = 0; q < npts; ++q) {
        const double* x0 = xi + (size_t)q * D;
        double Uq[BOSSS_MAX_VARS], Gq[BOSSS_MAX_VARS][3];
        for (int f = 0; f < nd; ++f) {
            int k = P.op.domain_degree[f], Np = P.dom_np[f];
            double v = 0, gr[3] = {0, 0, 0};
            for (int n = 0; n < Np; ++n) {
                double pv, pg[3];
                poly_eval(P.basis[k][n], D, x0, pv, pg);
                double cf = U[(long)j * Nd + P.dom_off[f] + n];
                v += cf * pv;
                for (int d = 0; d < D; ++d) gr[d] += cf * pg[d];
            }
            Uq[f] = v * P.scaling;
            for (int d = 0; d < D; ++d) Gq[f][d] = gr[d] * P.scaling * 2.0 / P.h[d];
        }
        double x[3];
        for (int d = 0; d < D; ++d) x[d] = c[d] + 0.5 * P.h[d] * x0[d];
        for (int e = 0; e < nc; ++e) {
            double fV = 0, fG[3] = {0, 0, 0};
            for (int ci = 0; ci < P.op.n_components; ++ci)
                if (P.op.components[ci].codomain == e) volume_terms<double>(P, P.op.components[ci], Uq, Gq, x, fV, fG);
            int k = P.op.codomain_degree[e], Np = P.cod_np[e];
            for (int m = 0; m < Np; ++m) {
                double pv, pg[3];
                poly_eval(P.basis[k][m], D, x0, pv, pg);
                double acc = fV * pv;
                for (int d = 0; d < D; ++d) acc += fG[d] * pg[d] * 2.0 / P.h[d];
                R[P.cod_off[e] + m] += w[q] * P.detJ * P.scaling * acc;
            }
        }
    }
}

// Face integral between jin (IN, lower cell, its face xi_d = +1) and jout (OUT, xi_d = -1),
// or a boundary face of jin (jout < 0, outward normal sgn*e_d, face xi_d = sgn); face
// nodes t[npts*(D-1)] in the in-plane directions (ascending), weights w.
static void face_integral(const Problem& P, int jin, int jout, int d, double sgn, int npts, const double* t,
                          const double* w, const double* U, double* Rin, double* Rout) {
    const int D = P.D, nd = P.op.n_domain, nc = P.op.n_codomain, Nd = P.dom_per_cell;
    int oth[2], no = 0;
    for (int d2 = 0; d2 < D; ++d2)
        if (d2 != d) oth[no++] = d2;
    double cIn[3];
    cell_center(P, jin, cIn);
    double nrm[3] = {0, 0, 0};
    nrm[d] = (jout >= 0) ? 1.0 : sgn;
    for (int q = 0; q < npts; ++q) {
        double xiIn[3], xiOut[3], x[3];
        xiIn[d] = (jout >= 0) ? 1.0 : sgn;
        xiOut[d] = -1.0;
        for (int k = 0; k < D - 1; ++k) xiIn[oth[k]] = xiOut[oth[k]] = t[(size_t)q * (D - 1) + k];
        for (int d2 = 0; d2 < D; ++d2) x[d2] = cIn[d2] + 0.5 * P.h[d2] * xiIn[d2];
        double UA[BOSSS_MAX_VARS], GA[BOSSS_MAX_VARS][3], UB[BOSSS_MAX_VARS], GB[BOSSS_MAX_VARS][3];
        for (int side = 0; side < 2; ++side) {
            if (side == 1 && jout < 0) break;
            const int jc = side ? jout : jin;
            const double* xi = side ? xiOut : xiIn;
            for (int f = 0; f < nd; ++f) {
                int k = P.op.domain_degree[f], Np = P.dom_np[f];
                double v = 0, gr[3] = {0, 0, 0};
                for (int n = 0; n < Np; ++n) {
                    double pv, pg[3];
                    poly_eval(P.basis[k][n], D, xi, pv, pg);
                    double cf = U[(long)jc * Nd + P.dom_off[f] + n];
                    v += cf * pv;
                    for (int dd = 0; dd < D; ++dd) gr[dd] += cf * pg[dd];
                }
                double* Uo = side ? UB : UA;
                double(*Go)[3] = side ? GB : GA;
                Uo[f] = v * P.scaling;
                for (int dd = 0; dd < D; ++dd) Go[f][dd] = gr[dd] * P.scaling * 2.0 / P.h[dd];
            }
        }
        const double wq = w[q] * P.faceSG[d];
        for (int e = 0; e < nc; ++e) {
            double gA = 0, gB = 0, GAv[3] = {0, 0, 0}, GBv[3] = {0, 0, 0};
            for (int ci = 0; ci < P.op.n_components; ++ci) {
                const auto& cp = P.op.components[ci];
                if (cp.codomain != e) continue;
                if (jout >= 0) inner_edge_terms<double>(P, cp, jin, jout, UA, GA, UB, GB, nrm, gA, GAv, gB, GBv);
                else boundary_edge_terms<double>(P, cp, jin, UA, GA, nrm, x, nullptr, 0, gA, GAv);
            }
            int k = P.op.codomain_degree[e], Np = P.cod_np[e];
            for (int m = 0; m < Np; ++m) {
                double pv, pg[3];
                poly_eval(P.basis[k][m], D, xiIn, pv, pg);
                double acc = gA * pv;
                for (int dd = 0; dd < D; ++dd) acc += GAv[dd] * pg[dd] * 2.0 / P.h[dd];
                Rin[P.cod_off[e] + m] += wq * P.scaling * acc;
                if (jout >= 0) {
                    poly_eval(P.basis[k][m], D, xiOut, pv, pg);
                    double acc2 = gB * pv;
                    for (int dd = 0; dd < D; ++dd) acc2 += GBv[dd] * pg[dd] * 2.0 / P.h[dd];
                    Rout[P.cod_off[e] + m] += wq * P.scaling * acc2;
                }
            }
        }
    }
}

}  // namespace orc

// len (nullable): the species' cell length scales of the SIP penalty (CoefficientSet.CellLengthScales
// of the species, XLaplace.cs:104-113 and the base SIPLaplace.GetPenalty, ipLaplace.cs:131-141)
// in place of the uncut grid's
extern "C" int orc_xdg_evaluate(const bosss_op_desc* op, const bosss_grid_desc* g, const unsigned char* vol_flags,
                                const unsigned char* face_flags, int64_t n_items, const int64_t* info,
                                const int64_t* offs, const double* nodes, const double* weights, const double* len,
                                const double* U, double* out) {
    using namespace orc;
    Problem P;
    g_err = setup(P, op, g);
    if (!g_err.empty()) return BOSSS_ERR_BAD_ARG;
    if (len)
        for (int j = 0; j < P.J; ++j) P.cj[j] = 1.0 / len[j];
    const int D = P.D, J = P.J, Nc = P.cod_per_cell;
    // uncut cells and faces of the species: the standard rules, masked
    evaluate<double>(P, 1.0, 0.0, U, out, vol_flags, face_flags);
    // cut items with their own rules, per item into buffers, then added in item order
    std::vector<double> Rb((size_t)n_items * Nc, 0.0), Ro((size_t)n_items * Nc, 0.0);
    std::vector<int> nbs(n_items, -1);
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t r = 0; r < n_items; ++r) {
        const int j = (int)info[r * 5 + 0], dim = (int)info[r * 5 + 1], d = (int)info[r * 5 + 2], s = (int)info[r * 5 + 3];
        const int64_t o0 = offs[r], o1 = offs[r + 1];
        const int npts = (int)(o1 - o0);
        std::vector<double> xi((size_t)npts * D), w(weights + o0, weights + o1);
        if (dim == D) {
            for (int q = 0; q < npts; ++q)
                for (int k = 0; k < D; ++k) xi[(size_t)q * D + k] = nodes[(o0 + q) * 3 + k];
            vol_integral(P, j, npts, xi.data(), w.data(), U, &Rb[(size_t)r * Nc]);
        } else {
            for (int q = 0; q < npts; ++q)
                for (int k = 0; k < D - 1; ++k) xi[(size_t)q * (D - 1) + k] = nodes[(o0 + q) * 3 + k];
            const int nb = neighbour(P, j, d, s);
            nbs[r] = nb;
            face_integral(P, j, nb, d, s ? 1.0 : -1.0, npts, xi.data(), w.data(), U, &Rb[(size_t)r * Nc],
                          &Ro[(size_t)r * Nc]);
        }
    }
    for (int64_t r = 0; r < n_items; ++r) {
        const int j = (int)info[r * 5 + 0];
        for (int i = 0; i < Nc; ++i) out[(size_t)j * Nc + i] += Rb[(size_t)r * Nc + i];
        if (nbs[r] >= 0)
            for (int i = 0; i < Nc; ++i) out[(size_t)nbs[r] * Nc + i] += Ro[(size_t)r * Nc + i];
    }
    (void)J;
    return 0;
}


using namespace orc;

extern "C" {

int orc_last_error(char* buf, size_t len) {
    if (len) {
        std::strncpy(buf, g_err.c_str(), len - 1);
        buf[len - 1] = 0;
    }
    return 0;
}

int orc_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

int orc_sizes(const bosss_op_desc* op, const bosss_grid_desc* g, int64_t* ndom, int64_t* ncod, int32_t* nq) {
    Problem P;
    g_err = setup(P, op, g);
    if (!g_err.empty()) return BOSSS_ERR_BAD_ARG;
    *ndom = (int64_t)P.J * P.dom_per_cell;
    *ncod = (int64_t)P.J * P.cod_per_cell;
    *nq = P.nQ1;
    return 0;
}

int orc_gauss_rule(int n, double* nodes, double* weights) {
    std::vector<double> x, w;
    gauss_legendre(n, x, w);
    for (int i = 0; i < n; ++i) { nodes[i] = x[i]; weights[i] = w[i]; }
    return 0;
}

// Monomial table of the orthonormal basis: for each polynomial, up to (k+1)^D terms;
// coef[p*T + t], exps[(p*T + t)*3 + d], T = (k+1)^D (unused slots have coef 0).
int orc_basis_monomials(int D, int k, double* coef, int32_t* exps) {
    auto B = make_basis(D, k);
    int T = 1;
    for (int d = 0; d < D; ++d) T *= (k + 1);
    for (size_t p = 0; p < B.size(); ++p)
        for (int t = 0; t < T; ++t) {
            bool have = t < (int)B[p].coef.size();
            coef[p * T + t] = have ? B[p].coef[t] : 0.0;
            for (int d = 0; d < 3; ++d) exps[(p * T + t) * 3 + d] = have ? B[p].exps[t][d] : 0;
        }
    return (int)B.size();
}

// phi[p*npts + i], dphi[(p*npts + i)*D + d] at reference points pts[i*D + d]
int orc_basis_eval(int D, int k, int npts, const double* pts, double* phi, double* dphi) {
    auto B = make_basis(D, k);
    for (size_t p = 0; p < B.size(); ++p)
        for (int i = 0; i < npts; ++i) {
            double v, g[3];
            poly_eval(B[p], D, pts + i * D, v, g);
            phi[p * npts + i] = v;
            if (dphi)
                for (int d = 0; d < D; ++d) dphi[(p * npts + i) * D + d] = g[d];
        }
    return (int)B.size();
}

// setup plus the boundary-state table (bnd may be null unless a component needs it)
static thread_local const int* g_kinds = nullptr;   // set by orc_set_boundary_kinds

static int setup_bnd(Problem& P, const bosss_op_desc* op, const bosss_grid_desc* g, const double* bnd) {
    g_err = setup(P, op, g);
    if (!g_err.empty()) return BOSSS_ERR_BAD_ARG;
    P.bnd = bnd;
    P.kinds = g_kinds;
    bool need_table = true;
    if (g_kinds) {
        need_table = false;
        for (long long i = 0; i < P.n_bnd_nodes; ++i) need_table = need_table || g_kinds[i] == 0;
    }
    if (!bnd && P.n_bnd_nodes > 0 && need_table)
        for (int c = 0; c < op->n_components; ++c)
            if (op->components[c].type == ORC_COMP_CNS_SIPG_MOMENTUM || op->components[c].type == ORC_COMP_CNS_SIPG_ENERGY ||
                op->components[c].type == BOSSS_COMP_HLLC_DENSITY_FLUX ||
                op->components[c].type == BOSSS_COMP_HLLC_MOMENTUM_FLUX ||
                op->components[c].type == BOSSS_COMP_HLLC_ENERGY_FLUX) {
                g_err = "CNS SIPG and HLLC on a grid with boundary faces need the boundary-state table";
                return BOSSS_ERR_BAD_ARG;
            }
    return 0;
}

// boundary-condition kinds of the boundary face nodes for the following calls (null: all 0;
// the array must stay alive until the next call)
int orc_set_boundary_kinds(const int* kinds) {
    g_kinds = kinds;
    return 0;
}

// number of boundary face nodes (rows of the boundary-state table)
int orc_boundary_nodes(const bosss_op_desc* op, const bosss_grid_desc* g, int64_t* n) {
    Problem P;
    g_err = setup(P, op, g);
    if (!g_err.empty()) return BOSSS_ERR_BAD_ARG;
    *n = P.n_bnd_nodes;
    return 0;
}

int orc_evaluate(const bosss_op_desc* op, const bosss_grid_desc* g, const double* bnd, double alpha, double beta,
                 const double* U, double* out) {
    Problem P;
    if (int rc = setup_bnd(P, op, g, bnd)) return rc;
    evaluate<double>(P, alpha, beta, U, out);
    return 0;
}

// exact adjoint product J(U)^T W
int orc_vjp(const bosss_op_desc* op, const bosss_grid_desc* g, const double* bnd, const double* U, const double* W,
            double* JTW) {
    Problem P;
    if (int rc = setup_bnd(P, op, g, bnd)) return rc;
    const int need = 2 * P.op.n_domain * (1 + P.D);
    if (need <= 8) vjp<8>(P, U, W, JTW);
    else if (need <= 24) vjp<24>(P, U, W, JTW);
    else if (need <= 40) vjp<40>(P, U, W, JTW);
    else vjp<2 * BOSSS_MAX_VARS * 4>(P, U, W, JTW);
    return 0;
}

// BlockMsrMatrix.SpMV (BlockMsrMatrix.cs:2554-2990): y = beta*y + alpha*A*x on a block-CSR
// matrix, blocks dense row-major (row_block x col_block), block rows in parallel.
int orc_bsr_spmv(int64_t nbr, int32_t br, int32_t bc, const int64_t* rowptr, const int32_t* colidx,
                 const double* vals, double alpha, const double* x, double beta, double* y) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nbr; ++i) {
        double acc[64];
        for (int r = 0; r < br; ++r) acc[r] = 0.0;
        for (int64_t b = rowptr[i]; b < rowptr[i + 1]; ++b) {
            const double* blk = vals + b * (int64_t)br * bc;
            const double* xb = x + (int64_t)colidx[b] * bc;
            for (int r = 0; r < br; ++r) {
                double s = 0.0;
                for (int c = 0; c < bc; ++c) s += blk[r * bc + c] * xb[c];
                acc[r] += s;
            }
        }
        for (int r = 0; r < br; ++r) {
            double& yr = y[i * br + r];
            yr = (beta == 0.0) ? alpha * acc[r] : beta * yr + alpha * acc[r];
        }
    }
    return 0;
}

// exact directional derivative J(U) V
int orc_jvp(const bosss_op_desc* op, const bosss_grid_desc* g, const double* bnd, const double* U, const double* V,
            double* JV) {
    Problem P;
    if (int rc = setup_bnd(P, op, g, bnd)) return rc;
    long nd = (long)P.J * P.dom_per_cell, nc = (long)P.J * P.cod_per_cell;
    std::vector<Dual> Ud(nd), od(nc);
    for (long i = 0; i < nd; ++i) Ud[i] = Dual(U[i], V[i]);
    evaluate<Dual>(P, 1.0, 0.0, Ud.data(), od.data());
    for (long i = 0; i < nc; ++i) JV[i] = od[i].d;
    return 0;
}

// Block-sparse Jacobian (self + face neighbours) at U, exact, by forward-mode over a
// distance-2 cell colouring. Output: for each cell row j, blocks in the order
// [self, (d=0,lower), (d=0,upper), (d=1,lower), ...]; missing neighbours get zero blocks.
// blocks[((j*(1+2D) + b)*Nc + row)*Nd + col]; nbr[j*(1+2D)+b] = column cell or -1.
int orc_jacobian_blocks(const bosss_op_desc* op, const bosss_grid_desc* g, const double* bnd, const double* U,
                        double* blocks, int32_t* nbr) {
    Problem P;
    if (int rc = setup_bnd(P, op, g, bnd)) return rc;
    const int D = P.D, J = P.J, Nd = P.dom_per_cell, Nc = P.cod_per_cell, NB = 1 + 2 * D;
    int m[3] = {1, 1, 1};
    for (int d = 0; d < D; ++d) {
        int n = P.g.n[d];
        if (!P.g.periodic[d]) m[d] = std::min(3, n);
        else {
            m[d] = n;  // fall back: every index its own colour
            for (int c = 3; c <= n; ++c)
                if (n % c == 0) { m[d] = c; break; }
        }
    }
    auto color = [&](int j) {
        int ijk[3];
        cell_ijk(P, j, ijk);
        int c = 0;
        for (int d = D - 1; d >= 0; --d) c = c * m[d] + (ijk[d] % m[d]);
        return c;
    };
    int ncol = 1;
    for (int d = 0; d < D; ++d) ncol *= m[d];
    for (int j = 0; j < J; ++j) {
        nbr[j * NB] = j;
        for (int d = 0; d < D; ++d)
            for (int s = 0; s < 2; ++s) nbr[j * NB + 1 + 2 * d + s] = neighbour(P, j, d, s);
    }
    std::memset(blocks, 0, sizeof(double) * (size_t)J * NB * Nc * Nd);
    std::vector<Dual> Ud((size_t)J * Nd), od((size_t)J * Nc);
    for (int c = 0; c < ncol; ++c)
        for (int col = 0; col < Nd; ++col) {
            for (int j = 0; j < J; ++j)
                for (int i = 0; i < Nd; ++i)
                    Ud[(size_t)j * Nd + i] = Dual(U[(size_t)j * Nd + i], (color(j) == c && i == col) ? 1.0 : 0.0);
            evaluate<Dual>(P, 1.0, 0.0, Ud.data(), od.data());
            for (int j = 0; j < J; ++j)
                for (int b = 0; b < NB; ++b) {
                    int jc = nbr[j * NB + b];
                    if (jc < 0 || color(jc) != c) continue;
                    // the first block with this column cell takes the entries (periodic n<3 may alias)
                    bool first = true;
                    for (int b2 = 0; b2 < b; ++b2)
                        if (nbr[j * NB + b2] == jc) first = false;
                    if (!first) continue;
                    for (int r = 0; r < Nc; ++r)
                        blocks[(((size_t)j * NB + b) * Nc + r) * Nd + col] = od[(size_t)j * Nc + r].d;
                }
        }
    return 0;
}

}  // extern "C"
