// dg_common.cuh -- shared device types of the DG evaluator: 1D basis tables,
// grid constants, forward-mode dual numbers and the mode-index maps of the
// reference's orthonormal polynomial ordering.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace bosss {

constexpr int KMAX = 4;   // highest DG degree with device kernels
constexpr int QMAX = 9;   // highest number of 1D Gauss nodes (order 17)

// 1D tables at the Gauss nodes of one rule: normalised Legendre polynomials
// L_a(x) = sqrt((2a+1)/2) P_a(x) and their derivatives. The D-dimensional basis of
// the reference (Square.cs / Cube_polynomials.cs) is the product L_a(x) L_b(y) L_c(z).
struct Tables1D {
    double A[QMAX][KMAX + 1];    // L_a(x_q)
    double dA[QMAX][KMAX + 1];   // L_a'(x_q)
    double w[QMAX];              // Gauss weights
    double xq[QMAX];             // Gauss nodes on [-1,1]
    double e[2][KMAX + 1];       // L_a(-1), L_a(+1)
    double de[2][KMAX + 1];      // L_a'(-1), L_a'(+1)
};

// Uniform Cartesian grid: every cell is the affine image x = c_j + (h/2) xi of [-1,1]^D.
struct GridConst {
    int D;
    int n[3];
    long long stride[3];     // cell index = sum_d ijk[d] * stride[d]
    int periodic[3];
    int J;                   // number of cells
    double lo[3], h[3];
    double twoh[3];          // 2/h_d  (InverseTransformation diagonal)
    double scaling;          // 1/sqrt(detJ)   (BasisData.cs:47-51)
    double detJ;             // prod h_d/2
    double faceSG[3];        // SqrtGramian of a face normal to d: prod_{d'!=d} h_d'/2
    // global grid of which this grid is a part (partitioned evaluation); equal to n, 0 and
    // periodic for a whole grid. Only the SIP cell length scale reads them.
    int gn[3], goff[3], gper[3];
};

__host__ __device__ constexpr int np_of(int D, int k) {
    return D == 2 ? (k + 1) * (k + 2) / 2 : (k + 1) * (k + 2) * (k + 3) / 6;
}

// index of the polynomial with exponents (a,b,c) (x,y,z) in the reference order:
// total degree ascending, then x-exponent ascending, then y-exponent ascending.
__host__ __device__ constexpr int mode3(int a, int b, int c) {
    return (a + b + c) * (a + b + c + 1) * (a + b + c + 2) / 6 + a * (a + b + c + 1) - a * (a - 1) / 2 + b;
}
__host__ __device__ constexpr int mode2(int a, int b) { return (a + b) * (a + b + 1) / 2 + a; }

// ------------------------------------------------------------------ dual numbers
// DualN<N>: value plus N tangent slots. N = 1 gives the JVP, N = (number of
// own-side inputs) gives the gradient of a scalar functional (VJP).
template <int N>
struct DualN {
    double v;
    double d[N];
    __host__ __device__ DualN() : v(0.0) {
#pragma unroll
        for (int i = 0; i < N; ++i) d[i] = 0.0;
    }
    __host__ __device__ DualN(double a) : v(a) {
#pragma unroll
        for (int i = 0; i < N; ++i) d[i] = 0.0;
    }
};

template <int N>
__host__ __device__ __forceinline__ DualN<N> operator+(const DualN<N>& a, const DualN<N>& b) {
    DualN<N> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <int N>
__host__ __device__ __forceinline__ DualN<N> operator-(const DualN<N>& a, const DualN<N>& b) {
    DualN<N> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <int N>
__host__ __device__ __forceinline__ DualN<N> operator-(const DualN<N>& a) {
    DualN<N> r;
    r.v = -a.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
    return r;
}
template <int N>
__host__ __device__ __forceinline__ DualN<N> operator*(const DualN<N>& a, const DualN<N>& b) {
    DualN<N> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <int N>
__host__ __device__ __forceinline__ DualN<N> operator/(const DualN<N>& a, const DualN<N>& b) {
    DualN<N> r;
    double inv = 1.0 / b.v;
    r.v = a.v * inv;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * inv;
    return r;
}
template <int N> __host__ __device__ __forceinline__ DualN<N> operator+(const DualN<N>& a, double b) { DualN<N> r = a; r.v += b; return r; }
template <int N> __host__ __device__ __forceinline__ DualN<N> operator+(double b, const DualN<N>& a) { DualN<N> r = a; r.v += b; return r; }
template <int N> __host__ __device__ __forceinline__ DualN<N> operator-(const DualN<N>& a, double b) { DualN<N> r = a; r.v -= b; return r; }
template <int N> __host__ __device__ __forceinline__ DualN<N> operator-(double b, const DualN<N>& a) { DualN<N> r = -a; r.v += b; return r; }
template <int N>
__host__ __device__ __forceinline__ DualN<N> operator*(const DualN<N>& a, double b) {
    DualN<N> r;
    r.v = a.v * b;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b;
    return r;
}
template <int N> __host__ __device__ __forceinline__ DualN<N> operator*(double b, const DualN<N>& a) { return a * b; }
template <int N>
__host__ __device__ __forceinline__ DualN<N> operator/(const DualN<N>& a, double b) { return a * (1.0 / b); }
template <int N>
__host__ __device__ __forceinline__ DualN<N> operator/(double a, const DualN<N>& b) {
    DualN<N> r;
    double inv = 1.0 / b.v;
    r.v = a * inv;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = -r.v * b.d[i] * inv;
    return r;
}
template <int N> __host__ __device__ __forceinline__ DualN<N>& operator+=(DualN<N>& a, const DualN<N>& b) { a = a + b; return a; }
template <int N> __host__ __device__ __forceinline__ DualN<N>& operator-=(DualN<N>& a, const DualN<N>& b) { a = a - b; return a; }
template <int N> __host__ __device__ __forceinline__ DualN<N>& operator*=(DualN<N>& a, const DualN<N>& b) { a = a * b; return a; }
template <int N> __host__ __device__ __forceinline__ DualN<N>& operator/=(DualN<N>& a, const DualN<N>& b) { a = a / b; return a; }
template <int N> __host__ __device__ __forceinline__ DualN<N>& operator+=(DualN<N>& a, double b) { a.v += b; return a; }
template <int N> __host__ __device__ __forceinline__ DualN<N>& operator-=(DualN<N>& a, double b) { a.v -= b; return a; }

template <int N>
__host__ __device__ __forceinline__ DualN<N> dsqrt(const DualN<N>& a) {
    DualN<N> r;
    r.v = sqrt(a.v);
    double s = 0.5 / r.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * s;
    return r;
}
__host__ __device__ __forceinline__ double dsqrt(double a) { return sqrt(a); }

__host__ __device__ __forceinline__ double pval(double a) { return a; }
template <int N> __host__ __device__ __forceinline__ double pval(const DualN<N>& a) { return a.v; }

}  // namespace bosss
