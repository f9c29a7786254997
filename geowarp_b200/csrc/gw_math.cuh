// Small dense math for per-particle work: 3x3 helpers, a forward-mode dual
// number, and a cyclic-Jacobi symmetric eigen-solver.  Everything is
// register-resident and templated on the scalar type.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#define GW_HD __host__ __device__ __forceinline__

namespace gw {
namespace {  // internal linkage: each translation unit compiles the kernels it launches

// ---------------------------------------------------------------- scalar helpers
GW_HD double val(double x) { return x; }
GW_HD float val(float x) { return x; }
// Elementary functions used by templated model code (g-prefixed so they do
// not collide with the C library overloads); Dual versions follow below.
GW_HD double gsqrt(double x) { return ::sqrt(x); }
GW_HD float gsqrt(float x) { return ::sqrtf(x); }
GW_HD double glog(double x) { return ::log(x); }
GW_HD float glog(float x) { return ::logf(x); }
GW_HD double gexp(double x) { return ::exp(x); }
GW_HD float gexp(float x) { return ::expf(x); }
GW_HD double gpow(double x, double p) { return ::pow(x, p); }
GW_HD float gpow(float x, float p) { return ::powf(x, p); }

template <typename R>
GW_HD R sq(R x) { return x * x; }

// ---------------------------------------------------------------- dual numbers
// Value plus N directional derivatives.  Used to differentiate the fixed-count
// local Newton iterations of the return maps exactly (the quantity Warp's tape
// differentiates in the reference) and to get the algorithmic tangent
// d tau_A / d e_trial_B.
template <int N, typename R>
struct Dual {
    R v;
    R d[N];
    GW_HD Dual() : v(0) {
#pragma unroll
        for (int i = 0; i < N; ++i) d[i] = 0;
    }
    GW_HD Dual(R x) : v(x) {
#pragma unroll
        for (int i = 0; i < N; ++i) d[i] = 0;
    }
    GW_HD Dual &operator+=(const Dual &o) { v += o.v; for (int i = 0; i < N; ++i) d[i] += o.d[i]; return *this; }
    GW_HD Dual &operator-=(const Dual &o) { v -= o.v; for (int i = 0; i < N; ++i) d[i] -= o.d[i]; return *this; }
    GW_HD Dual &operator*=(const Dual &o) {
        for (int i = 0; i < N; ++i) d[i] = d[i] * o.v + v * o.d[i];
        v *= o.v;
        return *this;
    }
};

template <int N, typename R> GW_HD R val(const Dual<N, R> &x) { return x.v; }

template <int N, typename R> GW_HD Dual<N, R> operator-(const Dual<N, R> &a) {
    Dual<N, R> r; r.v = -a.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
    return r;
}
template <int N, typename R> GW_HD Dual<N, R> operator+(const Dual<N, R> &a, const Dual<N, R> &b) {
    Dual<N, R> r; r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <int N, typename R> GW_HD Dual<N, R> operator-(const Dual<N, R> &a, const Dual<N, R> &b) {
    Dual<N, R> r; r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <int N, typename R> GW_HD Dual<N, R> operator*(const Dual<N, R> &a, const Dual<N, R> &b) {
    Dual<N, R> r; r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <int N, typename R> GW_HD Dual<N, R> operator/(const Dual<N, R> &a, const Dual<N, R> &b) {
    Dual<N, R> r; r.v = a.v / b.v;
    R ib = R(1) / b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
    return r;
}
// mixed scalar forms
template <int N, typename R> GW_HD Dual<N, R> operator+(const Dual<N, R> &a, R b) { Dual<N, R> r = a; r.v += b; return r; }
template <int N, typename R> GW_HD Dual<N, R> operator+(R b, const Dual<N, R> &a) { Dual<N, R> r = a; r.v += b; return r; }
template <int N, typename R> GW_HD Dual<N, R> operator-(const Dual<N, R> &a, R b) { Dual<N, R> r = a; r.v -= b; return r; }
template <int N, typename R> GW_HD Dual<N, R> operator-(R b, const Dual<N, R> &a) {
    Dual<N, R> r; r.v = b - a.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
    return r;
}
template <int N, typename R> GW_HD Dual<N, R> operator*(const Dual<N, R> &a, R b) {
    Dual<N, R> r; r.v = a.v * b;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b;
    return r;
}
template <int N, typename R> GW_HD Dual<N, R> operator*(R b, const Dual<N, R> &a) { return a * b; }
template <int N, typename R> GW_HD Dual<N, R> operator/(const Dual<N, R> &a, R b) { return a * (R(1) / b); }
template <int N, typename R> GW_HD Dual<N, R> operator/(R b, const Dual<N, R> &a) {
    Dual<N, R> r; r.v = b / a.v;
    R f = -r.v / a.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = f * a.d[i];
    return r;
}

template <int N, typename R> GW_HD Dual<N, R> gsqrt(const Dual<N, R> &a) {
    Dual<N, R> r; r.v = ::sqrt(a.v);
    R f = R(0.5) / r.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = f * a.d[i];
    return r;
}
template <int N, typename R> GW_HD Dual<N, R> glog(const Dual<N, R> &a) {
    Dual<N, R> r; r.v = ::log(a.v);
    R f = R(1) / a.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = f * a.d[i];
    return r;
}
template <int N, typename R> GW_HD Dual<N, R> gexp(const Dual<N, R> &a) {
    Dual<N, R> r; r.v = ::exp(a.v);
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = r.v * a.d[i];
    return r;
}
// a^p for constant p
template <int N, typename R> GW_HD Dual<N, R> gpow(const Dual<N, R> &a, R p) {
    Dual<N, R> r; r.v = ::pow(a.v, p);
    R f = p * ::pow(a.v, p - R(1));
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = f * a.d[i];
    return r;
}

// ---------------------------------------------------------------- generic small linear algebra
// Solve the 4x4 system M x = b by Gaussian elimination with partial pivoting
// on the value part; works for any scalar type with +,-,*,/.
template <typename T>
GW_HD void solve4(T M[4][4], T b[4], T x[4]) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        int piv = c;
        auto best = fabs(val(M[c][c]));
        for (int r = c + 1; r < 4; ++r) {
            auto a = fabs(val(M[r][c]));
            if (a > best) { best = a; piv = r; }
        }
        if (piv != c) {
            for (int k = 0; k < 4; ++k) { T t = M[c][k]; M[c][k] = M[piv][k]; M[piv][k] = t; }
            T t = b[c]; b[c] = b[piv]; b[piv] = t;
        }
        for (int r = c + 1; r < 4; ++r) {
            T f = M[r][c] / M[c][c];
            for (int k = c; k < 4; ++k) M[r][k] = M[r][k] - f * M[c][k];
            b[r] = b[r] - f * b[c];
        }
    }
    for (int r = 3; r >= 0; --r) {
        T s = b[r];
        for (int k = r + 1; k < 4; ++k) s = s - M[r][k] * x[k];
        x[r] = s / M[r][r];
    }
}

template <typename R>
GW_HD R det3(const R A[3][3]) {
    return A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) - A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
           A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
}

template <typename R>
GW_HD void inv3(const R A[3][3], R B[3][3]) {
    R d = det3(A);
    R id = R(1) / d;
    B[0][0] = (A[1][1] * A[2][2] - A[1][2] * A[2][1]) * id;
    B[0][1] = (A[0][2] * A[2][1] - A[0][1] * A[2][2]) * id;
    B[0][2] = (A[0][1] * A[1][2] - A[0][2] * A[1][1]) * id;
    B[1][0] = (A[1][2] * A[2][0] - A[1][0] * A[2][2]) * id;
    B[1][1] = (A[0][0] * A[2][2] - A[0][2] * A[2][0]) * id;
    B[1][2] = (A[0][2] * A[1][0] - A[0][0] * A[1][2]) * id;
    B[2][0] = (A[1][0] * A[2][1] - A[1][1] * A[2][0]) * id;
    B[2][1] = (A[0][1] * A[2][0] - A[0][0] * A[2][1]) * id;
    B[2][2] = (A[0][0] * A[1][1] - A[0][1] * A[1][0]) * id;
}

template <typename R>
GW_HD void matmul3(const R A[3][3], const R B[3][3], R C[3][3]) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) C[i][j] = A[i][0] * B[0][j] + A[i][1] * B[1][j] + A[i][2] * B[2][j];
}

// C = A B A^T
template <typename R>
GW_HD void congruence3(const R A[3][3], const R B[3][3], R C[3][3]) {
    R T[3][3];
    matmul3(A, B, T);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) C[i][j] = T[i][0] * A[j][0] + T[i][1] * A[j][1] + T[i][2] * A[j][2];
}

// ---------------------------------------------------------------- symmetric eigen-solver
// Cyclic Jacobi eigenvalue algorithm (Jacobi 1846; Golub & Van Loan, Matrix
// Computations, Alg. 8.5.2 with the stable rotation of Alg. 8.5.1).  On exit
// lam[k] are the eigenvalues and V[:, k] the eigenvectors (A = V diag V^T).
// Pairs whose off-diagonal entry is exactly zero are never rotated, so a
// block-diagonal (plane-strain) matrix keeps e_z as an exact eigenvector.
template <typename R>
GW_HD void eig_sym3(const R Ain[3][3], R lam[3], R V[3][3]) {
    R A[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) { A[i][j] = Ain[i][j]; V[i][j] = (i == j) ? R(1) : R(0); }
    const R eps = sizeof(R) == 8 ? R(1e-15) : R(1e-7);
    for (int sweep = 0; sweep < 12; ++sweep) {
        R off = fabs(A[0][1]) + fabs(A[0][2]) + fabs(A[1][2]);
        R dia = fabs(A[0][0]) + fabs(A[1][1]) + fabs(A[2][2]);
        if (off == R(0) || off <= eps * R(1e-3) * dia) break;
#pragma unroll
        for (int pq = 0; pq < 3; ++pq) {
            const int p = pq == 2 ? 1 : 0;
            const int q = pq == 0 ? 1 : 2;
            R apq = A[p][q];
            if (apq == R(0)) continue;
            R tau = (A[q][q] - A[p][p]) / (R(2) * apq);
            R t = (tau >= R(0) ? R(1) : R(-1)) / (fabs(tau) + ::sqrt(R(1) + tau * tau));
            R c = R(1) / ::sqrt(R(1) + t * t);
            R s = t * c;
            // A <- J^T A J with J_pp = J_qq = c, J_pq = s, J_qp = -s
#pragma unroll
            for (int k = 0; k < 3; ++k) {  // columns
                R akp = A[k][p], akq = A[k][q];
                A[k][p] = c * akp - s * akq;
                A[k][q] = s * akp + c * akq;
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) {  // rows
                R apk = A[p][k], aqk = A[q][k];
                A[p][k] = c * apk - s * aqk;
                A[q][k] = s * apk + c * aqk;
            }
            A[p][q] = A[q][p] = R(0);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                R vkp = V[k][p], vkq = V[k][q];
                V[k][p] = c * vkp - s * vkq;
                V[k][q] = s * vkp + c * vkq;
            }
        }
    }
    lam[0] = A[0][0];
    lam[1] = A[1][1];
    lam[2] = A[2][2];
}

}  // namespace
}  // namespace gw
