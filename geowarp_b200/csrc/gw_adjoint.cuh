// Adjoint of one 2D solid load step (vector-Jacobian products per particle).
//
// The reference differentiates only the last residual with its Warp tape
// (solvers/quasi_static_coupled_solver_3d.py:323-325).  The engine's adjoint is
// the total derivative of a load step: with u* solving R(u; q) = 0 for the
// particle inputs q = (x, lp, F_old, b_old, E),
//   q_bar = d(out)/dq^T out_bar + R_q^T lambda,   K^T lambda = d(out)/du^T out_bar,
// where out = (x_new, lp_new, F_new, b_new) are the G2P outputs
// (mpm/mpm_utils.py:1351-1419, mpm/gimp.py:428-462) and K = -dR/du the
// converged Jacobian.  Both VJPs are directional derivatives of one scalar,
// s = sum(output . weight) -- the G2P outputs weighted by their seeds, or the
// residual rows weighted by lambda -- with respect to 19 particle inputs:
//   inputs 0-1 x, 2-3 lp, 4-8 F_old (00,01,10,11,22), 9-12 b_old (00,01=10,11,22),
//   13 E, 14-17 H (00,01,10,11), 18 ubar_y (penalty footing).
// They come from one reverse-mode sweep per particle (solid2d_vjp): a forward
// pass over values, then the chain rule applied backwards through the same
// formulas as the forward kernels.  The principal-space constitutive update
// (eigen-solve and return map) enters through its Jacobian with respect to
// the trial b and E, evaluated once per particle (constitutive_jac).
#pragma once
#include "gw_step_kernels.cuh"

namespace gw {
namespace {  // internal linkage: each translation unit compiles the kernels it launches

constexpr int kAdjInputs = 19;
typedef Dual<2, double> AD;  // partials of the 1D shape functions in x and lp
constexpr int LX = 0, LLP = 2, LF = 4, LB = 9, LE = 13, LH = 14, LU = 18;

// cpGIMP axis with dual position and half-width; the cell indices come from
// the values (piecewise-constant), the weights carry the lanes.
GW_HD void gimp_axis_dual(const AD &xp, const AD &lp, double d, double inv_d, int &lower, int &span, AD w[3],
                          AD g[3]) {
    lower = cell_of(xp.v - lp.v, inv_d);
    const int upper = cell_of(xp.v + lp.v, inv_d);
    const int base = cell_of(xp.v, inv_d);
    if (upper == lower) {
        span = 2;
        AD fx = xp * inv_d - (double)base;
        w[0] = 1.0 - fx; w[1] = fx; w[2] = AD(0.0);
        g[0] = AD(-inv_d); g[1] = AD(inv_d); g[2] = AD(0.0);
    } else {
        span = 3;
        const double x0 = (double)lower * d, x1 = ((double)lower + 1.0) * d, x2 = ((double)lower + 2.0) * d;
        AD s0 = xp - x0, s2 = xp - x2;
        AD a0 = (s0.v < 0) ? -s0 : s0, a2 = (s2.v < 0) ? -s2 : s2;
        AD t0 = (lp + d) - a0, t2 = (lp + d) - a2;
        AD dl = lp * d;
        w[0] = t0 * t0 / (dl * 4.0);
        g[0] = (-t0 / (dl * 2.0) * s0) / a0;
        AD s1 = xp - x1;
        w[1] = 1.0 - (s1 * s1 + lp * lp) / (dl * 2.0);
        g[1] = -s1 / dl;
        w[2] = t2 * t2 / (dl * 4.0);
        g[2] = (-t2 / (dl * 2.0) * s2) / a2;
    }
}

// Isotropic tensor function f(b) = sum f_A(lambda) n_A n_A^T with dual lanes:
// fA carries the lanes of the principal values (through the return map), the
// off-diagonal lanes are D_AB (V^T db V)_AB with D_AB = (f_A - f_B)/(l_A - l_B)
// or its coalescence limit lim_AB.
template <int NL>
GW_HD void spectral_assemble(const double V[3][3], const double lamb[3], const Dual<NL, double> fA[3],
                             const double lim[3][3], const double dbp[][3][3], Dual<NL, double> out[3][3]) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double v = 0.0;
            for (int A = 0; A < 3; ++A) v += fA[A].v * V[i][A] * V[j][A];
            out[i][j] = Dual<NL, double>(v);
        }
    double D[3][3];
    for (int A = 0; A < 3; ++A)
        for (int B = 0; B < 3; ++B) {
            if (A == B) { D[A][B] = 0.0; continue; }
            const double dl = lamb[A] - lamb[B];
            const double sc = fmax(fabs(lamb[A]), fabs(lamb[B]));
            D[A][B] = (fabs(dl) > 1e-9 * sc) ? (fA[A].v - fA[B].v) / dl : lim[A][B];
        }
    for (int l = 0; l < NL; ++l) {
        double M[3][3];
        for (int A = 0; A < 3; ++A)
            for (int B = 0; B < 3; ++B) M[A][B] = (A == B) ? fA[A].d[l] : D[A][B] * dbp[l][A][B];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double v = 0.0;
                for (int A = 0; A < 3; ++A)
                    for (int B = 0; B < 3; ++B) v += V[i][A] * M[A][B] * V[j][B];
                out[i][j].d[l] = v;
            }
    }
}

// Principal return map of the principal-space models (Hencky, J2,
// Drucker-Prager) with its algorithmic tangent: lanes 0..2 seed the trial
// principal log strains, lane 3 seeds E (through lam and mu).
template <int MODEL>
GW_HD void principal_tangent_E(const LaunchConst &c, int model, double Ev, const double etr_v[3], double tau_v[3],
                               double dtau[3][4], double e_v[3], double de[3][4]) {
    typedef Dual<4, double> T;
    const double nu = c.nu;
    T E(Ev);
    E.d[3] = 1.0;
    const T lam = E * (nu / ((1.0 + nu) * (1.0 - 2.0 * nu)));
    const T mu = E * (1.0 / (2.0 * (1.0 + nu)));
    T etr[3], e[3], tau[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        etr[i] = T(etr_v[i]);
        etr[i].d[i] = 1.0;
    }
    if (model == GW_MODEL_J2) rm_j2<T, double, T>(etr, lam, mu, c.mc.kappa, e);
    else if (model == GW_MODEL_DP) rm_dp<T, double, T>(etr, lam, mu, c.mc, e);
    else
        for (int i = 0; i < 3; ++i) e[i] = etr[i];
    tau_hencky(e, lam, mu, tau);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        tau_v[i] = tau[i].v;
        e_v[i] = e[i].v;
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            dtau[i][l] = tau[i].d[l];
            de[i][l] = e[i].d[l];
        }
    }
}

// Jacobian of the principal-space constitutive update of one particle,
// evaluated once per particle: tau and b_new (plane-strain components 00,
// 01 = 10, 11, 22) with respect to the trial b's components (00, 01 = 10,
// 11, 22; a symmetric perturbation of the 01 / 10 pair) and E.  The trial b
// is eigen-decomposed once, each direction is rotated into its frame, the
// principal derivatives come from the return map's algorithmic tangent, and
// the isotropic tensor functions are assembled back with their coalescence
// limits.  The reverse sweep takes tau's and b_new's adjoints back to the
// trial b and E through this record, so the eigen-solve and the return map
// run once per particle.
constexpr int kCJ = 5;
struct ConstJac {
    double tv[4], Jt[4][kCJ];  // tau
    double bv[4], Jb[4][kCJ];  // b_new (G2P adjoint only)
};

template <int MODEL>
GW_HD void constitutive_jac(const LaunchConst &c, int model, const double B[3][3], double Ev, bool want_b,
                            ConstJac &cj) {
    typedef Dual<kCJ, double> CD;
    double lamb[3], V[3][3], Bc[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Bc[i][j] = B[i][j];
    eig_sym3(Bc, lamb, V);
    // directions 0..3: unit symmetric perturbations of b_trial 00, 01/10, 11, 22, rotated: V^T dB V
    double dbp[kCJ][3][3];
    const int pi[4] = {0, 0, 1, 2}, pj[4] = {0, 1, 1, 2};
    for (int k = 0; k < kCJ; ++k)
        for (int A = 0; A < 3; ++A)
            for (int Bq = 0; Bq < 3; ++Bq) {
                double v = 0.0;
                if (k < 4) {
                    const int i = pi[k], j = pj[k];
                    v = V[i][A] * V[j][Bq];
                    if (i != j) v += V[j][A] * V[i][Bq];
                }
                dbp[k][A][Bq] = v;
            }
    double etr_v[3], tv[3], dtau[3][4], ev[3], de[3][4];
    bool ok[3];
    for (int A = 0; A < 3; ++A) {
        ok[A] = lamb[A] > 1e-8;
        etr_v[A] = 0.5 * ::log(ok[A] ? lamb[A] : 1e-8);
    }
    principal_tangent_E<MODEL>(c, model, Ev, etr_v, tv, dtau, ev, de);
    CD fA[3], fB[3];
    double limT[3][3], limB[3][3];
    for (int A = 0; A < 3; ++A) {
        const double fb = ::exp(2.0 * ev[A]);
        fA[A] = CD(tv[A]);
        fB[A] = CD(fb);
        for (int k = 0; k < kCJ; ++k) {
            double dt = (k == 4) ? dtau[A][3] : 0.0, dl = (k == 4) ? de[A][3] : 0.0;
            for (int Bq = 0; Bq < 3; ++Bq) {
                const double detr = ok[Bq] ? dbp[k][Bq][Bq] / (2.0 * lamb[Bq]) : 0.0;
                dt += dtau[A][Bq] * detr;
                dl += de[A][Bq] * detr;
            }
            fA[A].d[k] = dt;
            fB[A].d[k] = 2.0 * fb * dl;
        }
        for (int Bq = 0; Bq < 3; ++Bq) {
            limT[A][Bq] = (dtau[A][A] - dtau[A][Bq]) / (2.0 * lamb[A]);
            limB[A][Bq] = 2.0 * fb * (de[A][A] - de[A][Bq]) / (2.0 * lamb[A]);
        }
    }
    CD out[3][3];
    spectral_assemble<kCJ>(V, lamb, fA, limT, dbp, out);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        cj.tv[k] = out[pi[k]][pj[k]].v;
        for (int l = 0; l < kCJ; ++l) cj.Jt[k][l] = out[pi[k]][pj[k]].d[l];
    }
    if (!want_b) return;
    spectral_assemble<kCJ>(V, lamb, fB, limB, dbp, out);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        cj.bv[k] = out[pi[k]][pj[k]].v;
        for (int l = 0; l < kCJ; ++l) cj.Jb[k][l] = out[pi[k]][pj[k]].d[l];
    }
}

// Weights of the contracted outputs: lambda per slot and field for the
// residual rows (zero on fixed DOFs), and / or the seeds of the G2P outputs.
struct VjpWeights {
    const double (*r)[2];           // [9][2] or null
    const double *x, *lp, *F, *b;   // G2P seeds ([2], [2], [9], [9]) or null
};

struct ParticleAdj {  // shape data of the particle's 9 slots, for the nodal adjoint
    int nid[9];
    double W[9], G[9][2];
    int lower[2], span[2];
    double xnew_dx[2];  // d lp_new_k / d x_new_k (clip branch: 0, +1 or -1)
};

// Reverse-mode VJP of one 2D solid particle: q[i] = ds / d input_i for the 19
// inputs, with s = sum(output . weight).  One forward pass
// keeps the values (and the 1D shape functions' partials in x and lp, from a
// 2-lane dual evaluation per axis); the sweep then applies the chain rule
// backwards through the same formulas: G2P outputs, residual rows, penalty,
// stress (principal-space models through the constitutive Jacobian cj;
// neo-Hookean and linear in closed form), F_new = f F_old, b_trial = f b_old
// f^T, f^-1, f = I + H, the gathered H / ubar / dx, and the shape functions.
// Nothing is recomputed per input, so the particle's state stays in registers.
template <int MODEL>
__device__ __forceinline__ void solid2d_vjp(const LaunchConst &c, const double *xv, const double *lpv,
                                            const double *Fo_v, const double *bo_v, double Ev, const double fext[2],
                                            const double du[9][2], const VjpWeights &wt, const ConstJac &cj,
                                            double q[kAdjInputs], ParticleAdj &o) {
    const gw_grid_t &g = c.g;
    const bool want_g2p = wt.x != nullptr;
    const int model = MODEL >= 0 ? MODEL : c.mc.model;
    const bool spectral = model == GW_MODEL_HENCKY || model == GW_MODEL_J2 || model == GW_MODEL_DP;
    const double nu = c.nu;
    const double cl = nu / ((1.0 + nu) * (1.0 - 2.0 * nu)), cm = 1.0 / (2.0 * (1.0 + nu));
    const double lam = Ev * cl, mu = Ev * cm;

    // ---------------- forward values
    double w[2][3], gw[2][3], dw[2][3][2], dgw[2][3][2];  // [axis][node], partials [d/dx, d/dlp]
    for (int k = 0; k < 2; ++k) {
        AD xd(xv[k]), ld(lpv[k]);
        xd.d[0] = 1.0;
        ld.d[1] = 1.0;
        AD wd[3], gd[3];
        gimp_axis_dual(xd, ld, g.h[k], g.inv_h[k], o.lower[k], o.span[k], wd, gd);
        for (int i = 0; i < 3; ++i) {
            w[k][i] = wd[i].v;
            gw[k][i] = gd[i].v;
            dw[k][i][0] = wd[i].d[0];
            dw[k][i][1] = wd[i].d[1];
            dgw[k][i][0] = gd[i].d[0];
            dgw[k][i][1] = gd[i].d[1];
        }
    }
    for (int a = 0; a < 9; ++a) {
        const int i = a % 3, j = a / 3;
        o.W[a] = w[0][i] * w[1][j];
        o.G[a][0] = gw[0][i] * w[1][j];
        o.G[a][1] = w[0][i] * gw[1][j];
        const int cx = o.lower[0] + i, cy = o.lower[1] + j;
        o.nid[a] = (cx >= 0 && cx <= g.n_grid[0] && cy >= 0 && cy <= g.n_grid[1]) ? cx + cy * (g.n_grid[0] + 1) : -1;
    }
    double H[2][2] = {{0.0, 0.0}, {0.0, 0.0}}, ubar = 0.0, dxp[2] = {0.0, 0.0};
    for (int a = 0; a < 9; ++a) {
        if (o.nid[a] < 0) continue;
        for (int k = 0; k < 2; ++k)
            for (int l = 0; l < 2; ++l) H[k][l] += o.G[a][k] * du[a][l];
        ubar += o.W[a] * du[a][1];
        dxp[0] += o.W[a] * du[a][0];
        dxp[1] += o.W[a] * du[a][1];
    }
    double Fi[3][3] = {{1.0 + H[0][0], H[0][1], 0.0}, {H[1][0], 1.0 + H[1][1], 0.0}, {0.0, 0.0, 1.0}};
    const double det2 = Fi[0][0] * Fi[1][1] - Fi[0][1] * Fi[1][0];
    const double Finv[2][2] = {{Fi[1][1] / det2, -Fi[0][1] / det2}, {-Fi[1][0] / det2, Fi[0][0] / det2}};
    double Fo[3][3], bo[3][3], Fn[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) { Fo[i][j] = Fo_v[i * 3 + j]; bo[i][j] = bo_v[i * 3 + j]; }
    matmul3(Fi, Fo, Fn);
    const double J = det3(Fn);
    double tau[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
    double lnJ = 0.0, eps[3][3], tr = 0.0, sg[3][3];
    if (spectral) {
        tau[0][0] = cj.tv[0];
        tau[0][1] = tau[1][0] = cj.tv[1];
        tau[1][1] = cj.tv[2];
        tau[2][2] = cj.tv[3];
    } else if (model == GW_MODEL_NEOHOOKEAN) {
        lnJ = ::log(J);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                const double ff = Fn[i][0] * Fn[j][0] + Fn[i][1] * Fn[j][1] + Fn[i][2] * Fn[j][2];
                tau[i][j] = mu * (ff - (i == j ? 1.0 : 0.0));
                if (i == j) tau[i][j] += lam * lnJ;
            }
    } else {
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) eps[i][j] = (Fn[i][j] + Fn[j][i]) * 0.5 - (i == j ? 1.0 : 0.0);
        tr = eps[0][0] + eps[1][1] + eps[2][2];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                sg[i][j] = mu * 2.0 * eps[i][j];
                if (i == j) sg[i][j] += lam * tr;
                tau[i][j] = J * sg[i][j];
            }
    }
    const double V0 = c.st.p_vol;
    const double ramp = (c.st.current_step + 1.0) / c.st.total_steps;
    const double gv = -c.st.gravity_mag * (c.st.gravity_full ? 1.0 : ramp);
    bool pen_on = false;
    double pen = 0.0, height = 0.0, pa = 0.0, sgn = 1.0;
    if (c.st.has_footing) {
        height = c.st.footing_initial_height + (c.st.current_step + 1.0) * c.st.footing_incr_disp;
        if (xv[1] >= height && xv[0] > c.st.footing_min[0] && xv[0] < c.st.footing_max[0]) {
            pa = c.st.penalty_factor * (c.g.h[0] / c.st.PPD);
            sgn = c.st.footing_stable ? -1.0 : 1.0;
            pen = sgn * (xv[1] + ubar - height) * (Ev * pa);
            pen_on = true;
        }
    }

    // ---------------- reverse sweep
    double xb[2] = {0.0, 0.0}, lpb[2] = {0.0, 0.0}, Eb = 0.0, ubarb = 0.0, dxb[2] = {0.0, 0.0}, penb = 0.0;
    double Fnb[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
    double Btb[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
    double taub[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
    double Wb[9], Gb[9][2], Finvb[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
    for (int a = 0; a < 9; ++a) { Wb[a] = 0.0; Gb[a][0] = Gb[a][1] = 0.0; }
    if (want_g2p) {  // x_new = x + dx ; lp_new from F_new's columns (clipped) ; F_new
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) Fnb[i][j] += wt.F[i * 3 + j];
        for (int k = 0; k < 2; ++k) {
            const double xn = xv[k] + dxp[k];
            const double U = ::sqrt(Fn[0][k] * Fn[0][k] + Fn[1][k] * Fn[1][k] + Fn[2][k] * Fn[2][k]);
            double v = U * c.st.lp0;
            int br = 0;
            if (xn - v < c.g.domain_min[k]) { v = xn - (c.g.domain_min[k] + 1e-6); br = 1; }
            if (xn + v > c.g.domain_max[k]) { v = (c.g.domain_max[k] - 1e-6) - xn; br = 2; }
            double xnb = wt.x[k];
            const double vb = wt.lp[k];
            if (br == 0) {
                const double Ub = vb * c.st.lp0;
                for (int i = 0; i < 3; ++i) Fnb[i][k] += Ub * Fn[i][k] / U;
            } else {
                xnb += br == 1 ? vb : -vb;
            }
            o.xnew_dx[k] = br == 0 ? 0.0 : (br == 1 ? 1.0 : -1.0);
            xb[k] += xnb;
            dxb[k] += xnb;
        }
    }
    if (wt.r)  // r_a = -(f^-T G_a) . tau V0 + W_a (rho V0 g + pen + f_ext)
        for (int a = 0; a < 9; ++a) {
            if (wt.r[a][0] == 0.0 && wt.r[a][1] == 0.0) continue;
            double wg[2], wgb[2] = {0.0, 0.0};
            for (int i = 0; i < 2; ++i) wg[i] = Finv[i][0] * o.G[a][0] + Finv[i][1] * o.G[a][1];
            for (int j = 0; j < 2; ++j) {
                const double lr = wt.r[a][j];
                wgb[0] -= tau[0][j] * V0 * lr;
                wgb[1] -= tau[1][j] * V0 * lr;
                taub[0][j] -= wg[0] * V0 * lr;
                taub[1][j] -= wg[1] * V0 * lr;
                double wc = fext[j];
                if (j == 1) wc += c.st.p_rho * V0 * gv;
                if (j == 1 && pen_on) {
                    wc += pen;
                    penb += o.W[a] * lr;
                }
                Wb[a] += wc * lr;
            }
            for (int m = 0; m < 2; ++m) {
                Gb[a][m] += wgb[0] * Finv[0][m] + wgb[1] * Finv[1][m];
                for (int i = 0; i < 2; ++i) Finvb[i][m] += wgb[i] * o.G[a][m];
            }
        }
    if (pen_on) {  // pen = sgn (x1 + ubar - height) E pa
        xb[1] += sgn * Ev * pa * penb;
        ubarb += sgn * Ev * pa * penb;
        Eb += sgn * (xv[1] + ubar - height) * pa * penb;
    }
    double Jb = 0.0;
    if (spectral) {  // tau, b_new from the constitutive Jacobian (components 00, 01 = 10, 11, 22)
        const double qb[4] = {taub[0][0], taub[0][1] + taub[1][0], taub[1][1], taub[2][2]};
        double pb[4] = {0.0, 0.0, 0.0, 0.0};
        if (want_g2p) {
            pb[0] = wt.b[0];
            pb[1] = wt.b[1] + wt.b[3];
            pb[2] = wt.b[4];
            pb[3] = wt.b[8];
        }
        double bc[5];
        for (int m = 0; m < kCJ; ++m) {
            double v = 0.0;
            for (int k = 0; k < 4; ++k) v += qb[k] * cj.Jt[k][m];
            if (want_g2p)
                for (int k = 0; k < 4; ++k) v += pb[k] * cj.Jb[k][m];
            bc[m] = v;
        }
        Btb[0][0] += bc[0];
        Btb[0][1] += 0.5 * bc[1];
        Btb[1][0] += 0.5 * bc[1];
        Btb[1][1] += bc[2];
        Btb[2][2] += bc[3];
        Eb += bc[4];
    } else {
        if (want_g2p)  // b_new = b_trial
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) Btb[i][j] += wt.b[i * 3 + j];
        double mub = 0.0, lamb = 0.0;
        if (model == GW_MODEL_NEOHOOKEAN) {  // tau = mu (F F^T - I) + lam ln J I
            for (int i = 0; i < 3; ++i)
                for (int k = 0; k < 3; ++k) {
                    double v = 0.0;
                    for (int j = 0; j < 3; ++j) v += (taub[i][j] + taub[j][i]) * Fn[j][k];
                    Fnb[i][k] += mu * v;
                }
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    const double ff = Fn[i][0] * Fn[j][0] + Fn[i][1] * Fn[j][1] + Fn[i][2] * Fn[j][2];
                    mub += taub[i][j] * (ff - (i == j ? 1.0 : 0.0));
                }
            const double trb = taub[0][0] + taub[1][1] + taub[2][2];
            lamb += lnJ * trb;
            Jb += lam * trb / J;
        } else {  // linear: tau = J (2 mu eps + lam tr(eps) I), eps = sym(F) - I
            double sgb[3][3], trs = 0.0;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    sgb[i][j] = J * taub[i][j];
                    Jb += taub[i][j] * sg[i][j];
                }
            for (int i = 0; i < 3; ++i) trs += sgb[i][i];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    mub += 2.0 * sgb[i][j] * eps[i][j];
                    const double eb = 2.0 * mu * sgb[i][j] + (i == j ? lam * trs : 0.0);
                    Fnb[i][j] += 0.5 * eb;
                    Fnb[j][i] += 0.5 * eb;
                }
            lamb += tr * trs;
        }
        Eb += mub * cm + lamb * cl;
    }
    if (Jb != 0.0) {  // d det(F) / dF = cofactor matrix
        Fnb[0][0] += Jb * (Fn[1][1] * Fn[2][2] - Fn[1][2] * Fn[2][1]);
        Fnb[0][1] += Jb * (Fn[1][2] * Fn[2][0] - Fn[1][0] * Fn[2][2]);
        Fnb[0][2] += Jb * (Fn[1][0] * Fn[2][1] - Fn[1][1] * Fn[2][0]);
        Fnb[1][0] += Jb * (Fn[0][2] * Fn[2][1] - Fn[0][1] * Fn[2][2]);
        Fnb[1][1] += Jb * (Fn[0][0] * Fn[2][2] - Fn[0][2] * Fn[2][0]);
        Fnb[1][2] += Jb * (Fn[0][1] * Fn[2][0] - Fn[0][0] * Fn[2][1]);
        Fnb[2][0] += Jb * (Fn[0][1] * Fn[1][2] - Fn[0][2] * Fn[1][1]);
        Fnb[2][1] += Jb * (Fn[0][2] * Fn[1][0] - Fn[0][0] * Fn[1][2]);
        Fnb[2][2] += Jb * (Fn[0][0] * Fn[1][1] - Fn[0][1] * Fn[1][0]);
    }
    // F_new = f F_old ; b_trial = f b_old f^T (b_old symmetric) ; f^-1
    double Fib[3][3], Fob[3][3], bob[3][3];
    {
        double S[3][3], T[3][3];  // S = Btb + Btb^T ; T = f b_old
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) S[i][j] = Btb[i][j] + Btb[j][i];
        matmul3(Fi, bo, T);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double v = 0.0;
                for (int k = 0; k < 3; ++k) v += Fnb[i][k] * Fo[j][k] + S[i][k] * T[k][j];
                Fib[i][j] = v;
                double u = 0.0;
                for (int k = 0; k < 3; ++k) u += Fi[k][i] * Fnb[k][j];
                Fob[i][j] = u;
            }
        double U2[3][3];  // f^T Btb f
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double v = 0.0;
                for (int k = 0; k < 3; ++k) v += Btb[i][k] * Fi[k][j];
                U2[i][j] = v;
            }
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double v = 0.0;
                for (int k = 0; k < 3; ++k) v += Fi[k][i] * U2[k][j];
                bob[i][j] = v;
            }
    }
    for (int i = 0; i < 2; ++i)  // d f^-1 = -f^-1 df f^-1
        for (int j = 0; j < 2; ++j) {
            double v = 0.0;
            for (int k = 0; k < 2; ++k)
                for (int m = 0; m < 2; ++m) v += Finv[k][i] * Finvb[k][m] * Finv[j][m];
            Fib[i][j] -= v;
        }
    // f = I + H ; H, ubar, dx gathered from the slots
    const double Hb[2][2] = {{Fib[0][0], Fib[0][1]}, {Fib[1][0], Fib[1][1]}};
    for (int a = 0; a < 9; ++a) {
        if (o.nid[a] < 0) continue;
        for (int k = 0; k < 2; ++k) Gb[a][k] += Hb[k][0] * du[a][0] + Hb[k][1] * du[a][1];
        Wb[a] += ubarb * du[a][1] + dxb[0] * du[a][0] + dxb[1] * du[a][1];
    }
    // W = w0 w1, G = (gw0 w1, w0 gw1) ; 1D weights -> x, lp
    double wb[2][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}}, gwb[2][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
    for (int a = 0; a < 9; ++a) {
        const int i = a % 3, j = a / 3;
        wb[0][i] += Wb[a] * w[1][j] + Gb[a][1] * gw[1][j];
        wb[1][j] += Wb[a] * w[0][i] + Gb[a][0] * gw[0][i];
        gwb[0][i] += Gb[a][0] * w[1][j];
        gwb[1][j] += Gb[a][1] * w[0][i];
    }
    for (int k = 0; k < 2; ++k)
        for (int i = 0; i < 3; ++i) {
            xb[k] += wb[k][i] * dw[k][i][0] + gwb[k][i] * dgw[k][i][0];
            lpb[k] += wb[k][i] * dw[k][i][1] + gwb[k][i] * dgw[k][i][1];
        }
    q[LX] = xb[0];
    q[LX + 1] = xb[1];
    q[LLP] = lpb[0];
    q[LLP + 1] = lpb[1];
    q[LF] = Fob[0][0];
    q[LF + 1] = Fob[0][1];
    q[LF + 2] = Fob[1][0];
    q[LF + 3] = Fob[1][1];
    q[LF + 4] = Fob[2][2];
    q[LB] = bob[0][0];
    q[LB + 1] = bob[0][1] + bob[1][0];
    q[LB + 2] = bob[1][1];
    q[LB + 3] = bob[2][2];
    q[LE] = Eb;
    q[LH] = Hb[0][0];
    q[LH + 1] = Hb[0][1];
    q[LH + 2] = Hb[1][0];
    q[LH + 3] = Hb[1][1];
    q[LU] = ubarb;
}

// ---------------------------------------------------------------- kernels
struct AdjState {  // per-particle adjoint arrays (user order)
    double *x, *lp, *F, *b, *E;  // [N*2], [N*2], [N*9], [N*9], [N]
};

// Nodal increments u_new - u_old of the particle's 9 slots (zero outside the grid).
__device__ __forceinline__ void gather_du(const LaunchConst &c, const PtrsP &p, int pid, const double *__restrict__ u_new,
                                          const double *__restrict__ u_old, double du[9][2]) {
    int lower[2];
    for (int k = 0; k < 2; ++k) lower[k] = cell_of(p.x[pid * 2 + k] - p.lp[pid * 2 + k], c.g.inv_h[k]);
    for (int a = 0; a < 9; ++a) {
        const int cx = lower[0] + a % 3, cy = lower[1] + a / 3;
        const bool in = cx >= 0 && cx <= c.g.n_grid[0] && cy >= 0 && cy <= c.g.n_grid[1];
        const int id = cx + cy * (c.g.n_grid[0] + 1);
        for (int l = 0; l < 2; ++l) du[a][l] = in ? u_new[(size_t)id * 2 + l] - u_old[(size_t)id * 2 + l] : 0.0;
    }
}

// Trial left Cauchy-Green tensor f b_old f^T of the particle (values), with
// f = I + H and H = sum_a du_a (x) grad N_a over the slots inside the grid:
// the values of the kinematics (gathered before the constitutive Jacobian).
__device__ __forceinline__ void trial_b(const LaunchConst &c, const double *xv, const double *lpv,
                                        const double *bo_v, const double du[9][2], double B[3][3]) {
    const gw_grid_t &g = c.g;
    Axis ax[2];
    for (int k = 0; k < 2; ++k) gimp_axis(xv[k], lpv[k], g.h[k], g.inv_h[k], ax[k]);
    double H[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
    for (int a = 0; a < 9; ++a) {
        const int i = a % 3, j = a / 3;
        const int cx = ax[0].lower + i, cy = ax[1].lower + j;
        if (!(cx >= 0 && cx <= g.n_grid[0] && cy >= 0 && cy <= g.n_grid[1])) continue;
        const double G0 = ax[0].gw[i] * ax[1].w[j], G1 = ax[0].w[i] * ax[1].gw[j];
        for (int l = 0; l < 2; ++l) {
            H[0][l] += G0 * du[a][l];
            H[1][l] += G1 * du[a][l];
        }
    }
    double f[3][3] = {{1.0 + H[0][0], H[0][1], 0.0}, {H[1][0], 1.0 + H[1][1], 0.0}, {0.0, 0.0, 1.0}};
    double bo[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) bo[i][j] = bo_v[i * 3 + j];
    congruence3(f, bo, B);
}

// q[i] = ds / d input_i for the particle's 19 inputs (external loads, E and the
// constitutive Jacobian gathered first).
template <int MODEL>
__device__ __forceinline__ void particle_vjp(const LaunchConst &c, const PtrsP &p, int pid, const double du[9][2],
                                             const VjpWeights &wt, double q[kAdjInputs], ParticleAdj &o) {
    const double E = p.E ? p.E[pid] : c.E0;
    const double ramp = (c.st.current_step + 1.0) / c.st.total_steps;
    const bool ext = p.ext_flag && p.ext_flag[pid];
    const double fext[2] = {ext ? c.st.point_load[0] * ramp : 0.0, ext ? c.st.point_load[1] * ramp : 0.0};
    ConstJac cj;
    const int model = MODEL >= 0 ? MODEL : c.mc.model;
    if (model == GW_MODEL_HENCKY || model == GW_MODEL_J2 || model == GW_MODEL_DP) {
        double B[3][3];
        trial_b(c, p.x + pid * 2, p.lp + pid * 2, p.b_old + (size_t)pid * 9, du, B);
        constitutive_jac<MODEL>(c, model, B, E, wt.x != nullptr, cj);
    }
    solid2d_vjp<MODEL>(c, p.x + pid * 2, p.lp + pid * 2, p.F_old + (size_t)pid * 9, p.b_old + (size_t)pid * 9, E, fext,
                       du, wt, cj, q, o);
}

// Adjoint G2P: seeds (x_new, lp_new, F_new, b_new) bars -> q_bar (written) and
// the nodal adjoint u_bar (free DOFs of active rows, atomically accumulated).
template <int MODEL>
__global__ void k_adjoint_g2p(LaunchConst c, PtrsP p, const double *__restrict__ u_new,
                              const double *__restrict__ u_old, const uint8_t *__restrict__ free_mask, PtrsA A,
                              AdjState seed_in, AdjState q_out, double *__restrict__ ubar_rows) {
    const int pid = blockIdx.x * blockDim.x + threadIdx.x;
    if (pid >= p.n) return;
    double du[9][2];
    gather_du(c, p, pid, u_new, u_old, du);
    VjpWeights wt;
    wt.r = nullptr;
    wt.x = seed_in.x + pid * 2;
    wt.lp = seed_in.lp + pid * 2;
    wt.F = seed_in.F + (size_t)pid * 9;
    wt.b = seed_in.b + (size_t)pid * 9;
    double q[kAdjInputs];
    ParticleAdj o;
    particle_vjp<MODEL>(c, p, pid, du, wt, q, o);
    double xb_eff[2];
    for (int k = 0; k < 2; ++k) xb_eff[k] = wt.x[k] + wt.lp[k] * o.xnew_dx[k];
    // particle-input adjoints
    q_out.x[pid * 2] = q[LX];
    q_out.x[pid * 2 + 1] = q[LX + 1];
    q_out.lp[pid * 2] = q[LLP];
    q_out.lp[pid * 2 + 1] = q[LLP + 1];
    double *Fq = q_out.F + (size_t)pid * 9, *bq = q_out.b + (size_t)pid * 9;
    for (int k = 0; k < 9; ++k) { Fq[k] = 0.0; bq[k] = 0.0; }
    Fq[0] = q[LF]; Fq[1] = q[LF + 1]; Fq[3] = q[LF + 2]; Fq[4] = q[LF + 3]; Fq[8] = q[LF + 4];
    bq[0] = q[LB]; bq[1] = 0.5 * q[LB + 1]; bq[3] = 0.5 * q[LB + 1]; bq[4] = q[LB + 2]; bq[8] = q[LB + 3];
    q_out.E[pid] = q[LE];
    // nodal adjoint: H_bar_kl G_b,k on component l, plus W_b x_bar_eff
    const double Hb[2][2] = {{q[LH], q[LH + 1]}, {q[LH + 2], q[LH + 3]}};
    for (int b = 0; b < 9; ++b) {
        const int id = o.nid[b];
        if (id < 0) continue;
        const uint8_t fm = free_mask[id];
        if (!fm) continue;
        const int row = A.node2row[id];
        if (!in_range(row, A.n_rows, GS_ADJOINT)) continue;
        for (int l = 0; l < 2; ++l) {
            if (!((fm >> l) & 1)) continue;
            const double v = Hb[0][l] * o.G[b][0] + Hb[1][l] * o.G[b][1] + o.W[b] * xb_eff[l];
            atomicAdd(&ubar_rows[(size_t)row * 2 + l], v);
        }
    }
}

// Adjoint P2G: q_bar += sum_a lambda_a . d r_a / d q over free DOFs.
template <int MODEL>
__global__ void k_adjoint_residual(LaunchConst c, PtrsP p, const double *__restrict__ u_new,
                                   const double *__restrict__ u_old, const uint8_t *__restrict__ free_mask, PtrsA A,
                                   const double *__restrict__ lambda_rows, AdjState q_out) {
    const int pid = blockIdx.x * blockDim.x + threadIdx.x;
    if (pid >= p.n) return;
    double du[9][2];
    gather_du(c, p, pid, u_new, u_old, du);
    // lambda of the particle's slots (zero on fixed DOFs and outside the grid)
    double lam_w[9][2];
    {
        int lower[2];
        for (int k = 0; k < 2; ++k) lower[k] = cell_of(p.x[pid * 2 + k] - p.lp[pid * 2 + k], c.g.inv_h[k]);
        for (int a = 0; a < 9; ++a) {
            lam_w[a][0] = lam_w[a][1] = 0.0;
            const int cx = lower[0] + a % 3, cy = lower[1] + a / 3;
            if (cx < 0 || cx > c.g.n_grid[0] || cy < 0 || cy > c.g.n_grid[1]) continue;
            const int id = cx + cy * (c.g.n_grid[0] + 1);
            const uint8_t fm = free_mask[id];
            if (!fm) continue;
            const int row = A.node2row[id];
            if (!in_range(row, A.n_rows, GS_ADJOINT)) continue;
            for (int f = 0; f < 2; ++f)
                if ((fm >> f) & 1) lam_w[a][f] = lambda_rows[(size_t)row * 2 + f];
        }
    }
    VjpWeights wt;
    wt.r = lam_w;
    wt.x = wt.lp = wt.F = wt.b = nullptr;
    double q[kAdjInputs];
    ParticleAdj o;
    particle_vjp<MODEL>(c, p, pid, du, wt, q, o);  // uses inputs x .. E
    q_out.x[pid * 2] += q[LX];
    q_out.x[pid * 2 + 1] += q[LX + 1];
    q_out.lp[pid * 2] += q[LLP];
    q_out.lp[pid * 2 + 1] += q[LLP + 1];
    double *Fq = q_out.F + (size_t)pid * 9, *bq = q_out.b + (size_t)pid * 9;
    Fq[0] += q[LF]; Fq[1] += q[LF + 1]; Fq[3] += q[LF + 2]; Fq[4] += q[LF + 3]; Fq[8] += q[LF + 4];
    bq[0] += q[LB]; bq[1] += 0.5 * q[LB + 1]; bq[3] += 0.5 * q[LB + 1]; bq[4] += q[LB + 2]; bq[8] += q[LB + 3];
    q_out.E[pid] += q[LE];
}

// A^T with the same (symmetric) block pattern: block (r, c) of A^T is the
// transpose of block (c, r) of A.
template <int D, typename VT>
__global__ void k_bsr_transpose(gw_grid_t g, PtrsA A, VT *__restrict__ AT) {
    const int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (r >= A.n_rows) return;
    const int lane = threadIdx.x & 31;
    const int nf = A.nf, node = A.row2node[r];
    if (!in_range(node, g.n_nodes, GS_TRANSPOSE)) return;
    int ic[3] = {0, 0, 0};
    {
        int q = node;
        for (int k = 0; k < D; ++k) { ic[k] = q % (g.n_grid[k] + 1); q /= (g.n_grid[k] + 1); }
    }
    const VT *vals = (const VT *)A.vals;
    for (int j = A.row_ptr[r] + lane; j < A.row_ptr[r + 1]; j += 32) {
        const int cr = A.cols[j];
        if (!in_range(cr, A.n_rows, GS_TRANSPOSE)) continue;
        const int cnode = A.row2node[cr];
        if (!in_range(cnode, g.n_nodes, GS_TRANSPOSE)) continue;
        int off[3] = {0, 0, 0}, q = cnode;
        bool ok = true;
        for (int k = 0; k < D; ++k) {
            off[k] = ic[k] - q % (g.n_grid[k] + 1);
            q /= (g.n_grid[k] + 1);
            ok = ok && in_range(off[k] + 2, 5, GS_TRANSPOSE);
        }
        if (!ok) continue;
        const int slot = stencil_slot(A.stencil, A.mw, cnode, offset_bit<D>(off));
        if (slot < 0 || !in_range((long long)A.row_ptr[cr] + slot, A.nnzb, GS_TRANSPOSE)) continue;
        const VT *src = vals + (size_t)j * nf * nf;
        VT *dst = AT + ((size_t)A.row_ptr[cr] + slot) * nf * nf;
        for (int f = 0; f < nf; ++f)
            for (int gg = 0; gg < nf; ++gg) dst[gg * nf + f] = src[f * nf + gg];
    }
}

}  // namespace
}  // namespace gw
