// Compiled CPU restatement of the oracle's per-particle work for the 2D solid
// kind with Hencky elasticity.  TEST INFRASTRUCTURE: only the tests and the
// benchmark's CPU-baseline and reference legs load it, never the product.
//
// It computes, per particle and in OpenMP threads over particles, exactly
// what oracle/mpm.py OracleEngine.local (solid2d branch, 'Hencky elasticity',
// no penalty footing) and the complex-step columns of OracleEngine.assemble
// compute with NumPy:
//   residual contributions r[a][f] of the particle's 3x3 nodes,
//     mpm/mpm_utils.py:416-596 (incremental F, trial b, principal Hencky
//     stress through eig3, internal force, gravity, point load);
//   the element tangent K = -dr/du by complex-step differentiation of r with
//     respect to each of the 18 local nodal unknowns (step 1e-30i, exact to
//     round-off), which replaces Warp's coloured reverse-mode sweeps
//     (solvers/sparse_differentiation.py:8-401) in the oracle;
//   F_new, b_new and the Cauchy stress of the converged-state bookkeeping.
// The symmetric 3x3 eigen-decomposition is the oracle's cyclic Jacobi method
// (oracle/eig.py: Jacobi 1846; Golub & Van Loan section 8.5), written so that
// it stays analytic in the matrix entries.  Shape functions, activation, the
// global assembly, the sparse direct solve and G2P stay in the NumPy oracle.
//
// Build: g++ -O3 -fopenmp -shared -fPIC (oracle/native.py builds it into
// oracle/_build/ when asked).
#include <cmath>
#include <complex>
#include <cstdint>

namespace {

typedef std::complex<double> cd;

inline double re(double v) { return v; }
inline double re(const cd &v) { return v.real(); }
inline double im(double) { return 0.0; }
inline double im(const cd &v) { return v.imag(); }

template <class T>
void eye3(T m[3][3]) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) m[i][j] = T(i == j ? 1.0 : 0.0);
}

// oracle/eig.py eigh3: 8 cyclic sweeps over the pairs (0,1), (0,2), (1,2)
template <class T>
void eigh3(const T Ain[3][3], T lam[3], T V[3][3]) {
    static const int P[3][2] = {{0, 1}, {0, 2}, {1, 2}};
    T A[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) A[i][j] = Ain[i][j];
    eye3(V);
    for (int sweep = 0; sweep < 8; ++sweep) {
        for (int pp = 0; pp < 3; ++pp) {
            const int p = P[pp][0], q = P[pp][1];
            const T apq = A[p][q];
            const T diff = A[p][p] - A[q][q];
            const bool nz = re(apq) != 0.0 || im(apq) != 0.0;
            const double dre = re(diff);
            T th;
            if (!nz) th = T(0.0);
            else if (dre != 0.0) th = -0.5 * std::atan(2.0 * apq / diff);  // tan 2t = -2 a_pq / (a_pp - a_qq)
            else th = T(re(apq) > 0.0 ? -M_PI / 4 : M_PI / 4);
            const T c = std::cos(th), s = std::sin(th);
            T G[3][3];
            eye3(G);
            G[p][p] = c;
            G[q][q] = c;
            G[p][q] = s;
            G[q][p] = -s;
            T GA[3][3], B[3][3], W[3][3];
            for (int i = 0; i < 3; ++i)  // G^T A
                for (int k = 0; k < 3; ++k) {
                    T v = T(0.0);
                    for (int j = 0; j < 3; ++j) v += G[j][i] * A[j][k];
                    GA[i][k] = v;
                }
            for (int i = 0; i < 3; ++i)  // (G^T A) G
                for (int l = 0; l < 3; ++l) {
                    T v = T(0.0);
                    for (int k = 0; k < 3; ++k) v += GA[i][k] * G[k][l];
                    B[i][l] = v;
                }
            B[p][q] = T(0.0);
            B[q][p] = T(0.0);
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) A[i][j] = B[i][j];
            for (int i = 0; i < 3; ++i)  // V G
                for (int l = 0; l < 3; ++l) {
                    T v = T(0.0);
                    for (int k = 0; k < 3; ++k) v += V[i][k] * G[k][l];
                    W[i][l] = v;
                }
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) V[i][j] = W[i][j];
        }
    }
    for (int i = 0; i < 3; ++i) lam[i] = A[i][i];
}

// sum_A vals[A] n_A n_A^T (oracle/eig.py from_principal)
template <class T>
void from_principal(const T vals[3], const T V[3][3], T out[3][3]) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            T v = T(0.0);
            for (int a = 0; a < 3; ++a) v += V[i][a] * vals[a] * V[j][a];
            out[i][j] = v;
        }
}

template <class T>
T det3(const T A[3][3]) {
    return A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) - A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
           A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
}

struct Particle {
    const double *W;     // [9]
    const double *Gr;    // [9][2] reference gradient weights
    const double *Uo;    // [9][2] previous nodal values
    const double *Fo;    // [3][3]
    const double *bo;    // [3][3]
    double lam, mu, p_vol, p_rho, gy;
    double fext[2];
};

// OracleEngine.local, solid2d branch, Hencky elasticity, for one particle
template <class T>
void local(const Particle &P, const T Un[9][2], T r[9][2], T Fn[3][3], T bn[3][3], T s3[3][3]) {
    T dU[9][2];
    for (int a = 0; a < 9; ++a)
        for (int k = 0; k < 2; ++k) dU[a][k] = Un[a][k] - P.Uo[a * 2 + k];
    T Hd[2][2] = {{T(0.0), T(0.0)}, {T(0.0), T(0.0)}};
    for (int k = 0; k < 2; ++k)
        for (int l = 0; l < 2; ++l)
            for (int a = 0; a < 9; ++a) Hd[k][l] += P.Gr[a * 2 + k] * dU[a][l];
    const T f00 = 1.0 + Hd[0][0], f01 = Hd[0][1], f10 = Hd[1][0], f11 = 1.0 + Hd[1][1];
    const T d = f00 * f11 - f01 * f10;
    const T Finv[2][2] = {{f11 / d, -f01 / d}, {-f10 / d, f00 / d}};
    T F3[3][3] = {{f00, f01, T(0.0)}, {f10, f11, T(0.0)}, {T(0.0), T(0.0), T(1.0)}};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            T v = T(0.0);
            for (int k = 0; k < 3; ++k) v += F3[i][k] * P.Fo[k * 3 + j];
            Fn[i][j] = v;
        }
    const T J = det3(Fn);
    T Fb[3][3], btr[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            T v = T(0.0);
            for (int k = 0; k < 3; ++k) v += F3[i][k] * P.bo[k * 3 + j];
            Fb[i][j] = v;
        }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            T v = T(0.0);
            for (int k = 0; k < 3; ++k) v += Fb[i][k] * F3[j][k];
            btr[i][j] = v;
        }
    T lamv[3], V[3][3];
    eigh3(btr, lamv, V);
    T e[3], taup[3], be[3];
    for (int a = 0; a < 3; ++a) e[a] = 0.5 * std::log(re(lamv[a]) > 1e-8 ? lamv[a] : T(1e-8));
    const T tr = e[0] + e[1] + e[2];
    for (int a = 0; a < 3; ++a) {
        taup[a] = P.lam * tr + 2.0 * P.mu * e[a];  // mpm/mpm_utils.py:541-542
        be[a] = std::exp(2.0 * e[a]);
    }
    T tau[3][3];
    from_principal(taup, V, tau);
    from_principal(be, V, bn);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) s3[i][j] = tau[i][j] / J;
    const T Vn = P.p_vol * J;
    const T rho = P.p_rho / J;
    for (int a = 0; a < 9; ++a) {
        T gg[2];
        for (int k = 0; k < 2; ++k) gg[k] = Finv[k][0] * P.Gr[a * 2 + 0] + Finv[k][1] * P.Gr[a * 2 + 1];
        for (int j = 0; j < 2; ++j) {
            const T g = T(j == 1 ? P.gy : 0.0);
            r[a][j] = (-(gg[0] * s3[0][j] + gg[1] * s3[1][j]) + P.W[a] * rho * g) * Vn + P.W[a] * P.fext[j];
        }
    }
}

}  // namespace

extern "C" {

// Per-particle residuals (and, with want_K, element tangents) of the 2D solid
// Hencky kind for N particles.  Arrays are C-contiguous FP64:
//   W[N][9], Gr[N][9][2], Un[N][9][2], Uo[N][9][2], F_old[N][3][3],
//   b_old[N][3][3], E[N], fext[N][2] (point load times the ramp);
//   gy: the vertical gravity acceleration of this load step (negative down).
// Outputs: r[N][9][2]; K[N][18][18] with K[n][a*2+f][b*2+g] = -d r[a][f] /
// d u[b][g] (when want_K); F_new, b_new, sigma [N][3][3].
// Returns 0, or -1 on bad arguments.
int gw_oracle_solid2d_hencky(int64_t N, const double *W, const double *Gr, const double *Un, const double *Uo,
                             const double *F_old, const double *b_old, const double *E, double nu, double p_vol,
                             double p_rho, double gy, const double *fext, int32_t want_K, int32_t threads, double *r,
                             double *K, double *F_new, double *b_new, double *sigma) {
    if (N < 0 || !W || !Gr || !Un || !Uo || !F_old || !b_old || !E || !fext || !r || !F_new || !b_new || !sigma ||
        (want_K && !K) || threads < 1)
        return -1;
    const double h = 1e-30;  // complex step (oracle/mpm.py CS_H)
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int64_t n = 0; n < N; ++n) {
        Particle P;
        P.W = W + n * 9;
        P.Gr = Gr + n * 18;
        P.Uo = Uo + n * 18;
        P.Fo = F_old + n * 9;
        P.bo = b_old + n * 9;
        P.lam = E[n] * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
        P.mu = E[n] / (2.0 * (1.0 + nu));
        P.p_vol = p_vol;
        P.p_rho = p_rho;
        P.gy = gy;
        P.fext[0] = fext[n * 2 + 0];
        P.fext[1] = fext[n * 2 + 1];
        double u[9][2], rr[9][2], Fn[3][3], bn[3][3], s3[3][3];
        for (int a = 0; a < 9; ++a)
            for (int k = 0; k < 2; ++k) u[a][k] = Un[n * 18 + a * 2 + k];
        local<double>(P, u, rr, Fn, bn, s3);
        for (int a = 0; a < 9; ++a)
            for (int k = 0; k < 2; ++k) r[n * 18 + a * 2 + k] = rr[a][k];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                F_new[n * 9 + i * 3 + j] = Fn[i][j];
                b_new[n * 9 + i * 3 + j] = bn[i][j];
                sigma[n * 9 + i * 3 + j] = s3[i][j];
            }
        if (!want_K) continue;
        cd uc[9][2], rc[9][2], Fc[3][3], bc[3][3], sc[3][3];
        for (int col = 0; col < 18; ++col) {
            for (int a = 0; a < 9; ++a)
                for (int k = 0; k < 2; ++k) uc[a][k] = cd(u[a][k], (a * 2 + k) == col ? h : 0.0);
            local<cd>(P, uc, rc, Fc, bc, sc);
            for (int a = 0; a < 9; ++a)
                for (int k = 0; k < 2; ++k) K[n * 324 + (a * 2 + k) * 18 + col] = -rc[a][k].imag() / h;
        }
    }
    return 0;
}

// Triplets of the global Jacobian from the element tangents: for every particle
// n, row (a, f) and column (b, g) whose DOFs are both free (ok[n][a*2+f]), the
// entry (dofs[n][a*2+f], dofs[n][b*2+g], K[n][a*2+f][b*2+g]), in the order
// n, (a, f), (b, g) -- the order in which the oracle's NumPy masks list them,
// so the summed matrix is the same.  offsets[n]: the first output slot of
// particle n (an exclusive prefix sum of the squared free-DOF counts).
int gw_oracle_triplets(int64_t N, const int64_t *dofs, const uint8_t *ok, const double *K, const int64_t *offsets,
                       int32_t threads, int64_t *rows, int64_t *cols, double *vals) {
    if (N < 0 || !dofs || !ok || !K || !offsets || !rows || !cols || !vals || threads < 1) return -1;
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int64_t n = 0; n < N; ++n) {
        int64_t o = offsets[n];
        for (int i = 0; i < 18; ++i) {
            if (!ok[n * 18 + i]) continue;
            for (int j = 0; j < 18; ++j) {
                if (!ok[n * 18 + j]) continue;
                rows[o] = dofs[n * 18 + i];
                cols[o] = dofs[n * 18 + j];
                vals[o] = K[n * 324 + i * 18 + j];
                ++o;
            }
        }
    }
    return 0;
}

}  // extern "C"
