// Per-particle residual and exact element tangent of the implicit cpGIMP step.
//
// The residual contributions of one particle to its 3^D local nodes depend on
// the nodal unknowns only through a short vector
//     theta = (H = sum_a G_a (x) du_a, pbar, grad~p, dp~, ubar_v)
// (H is the reference's delta_u_GRAD, mpm/mpm_utils.py:492-507; the pressure
// terms follow :929-950 and :1163-1194; ubar_v is the penalty footing
// displacement, :1242-1245).  Each residual row is linear in a short vector
// of stress-like quantities Q(theta):
//     r_a^u_j = -sum_i G_a,i Qu_ij + W_a g_j Qs + W_a [j = vert] Qpen + consts
//     r_a^p   =  W_a Qm1 + sum_i G_a,i Qm2_i + (W_a - Wavg_a) Qm3
// so the element matrix is K_ab = -Bhat_a^T (dQ/dtheta) B_b.  dQ/dtheta is
// formed once per particle: kinematics by hand, the eigen step of the
// Hencky-family models by the derivative of isotropic tensor functions
// (divided differences, with the coalescence limit), and the return maps by
// forward-mode duals through their fixed local iteration counts.  This replaces
// the reference's 50/75/500 coloured reverse-mode sweeps per Newton iteration
// (solvers/quasi_static_solver_2d.py:169-192, solvers/sparse_differentiation.py).
#pragma once
#include "gw_gimp.cuh"
#include "gw_models.cuh"

namespace gw {
namespace {  // internal linkage: each translation unit compiles the kernels it launches

template <int KIND> struct KindTraits;
template <> struct KindTraits<GW_KIND_SOLID2D> { static const int D = 2, NF = 2, NS = 9; static const bool UP = false; };
template <> struct KindTraits<GW_KIND_COUPLED2D> { static const int D = 2, NF = 3, NS = 9; static const bool UP = true; };
template <> struct KindTraits<GW_KIND_COUPLED3D> { static const int D = 3, NF = 4, NS = 27; static const bool UP = true; };

// Layout of Q and theta for a kind.
template <int KIND>
struct Layout {
    static const int D = KindTraits<KIND>::D;
    static const bool UP = KindTraits<KIND>::UP;
    // Q indices
    static const int QU = 0;                          // D*D
    static const int QS = D * D;                      // 1
    static const int QPEN = QS + 1;                   // 1
    static const int QM1 = QPEN + 1;                  // coupled only
    static const int QM2 = QM1 + 1;                   // D
    static const int QM3 = QM2 + D;                   // 1
    static const int NQ = UP ? QM3 + 1 : QPEN + 1;
    // theta indices
    static const int TH = 0;                          // D*D, index k*D + l
    static const int TU = D * D;                      // ubar_v
    static const int TP = TU + 1;                     // pbar
    static const int TG = TP + 1;                     // grad~p (D)
    static const int TD = TG + D;                     // dp~
    static const int NT = UP ? TD + 1 : TU + 1;
};

struct LaunchConst {
    gw_grid_t g;
    gw_step_t st;
    MatConst mc;
    double E0, nu;
};

// Mobility of the u-p mass balance at the current Jacobian J: the constant
// k0, or (law 1) Uzuoka & Borja (2012) Eq. 86,
//   k(J) = k0 (2 mu + lam) J / (mu (1 + J^-2) + (1 - ln J) lam J^-2),
// with its derivative dk/dJ for the tangent.
GW_HD double mobility_of(const gw_step_t &st, double J, double lam, double mu, double *dk_dJ) {
    if (st.mobility_law != 1) {
        if (dk_dJ) *dk_dJ = 0.0;
        return st.mobility;
    }
    const double iJ2 = 1.0 / (J * J);
    const double num = (2.0 * mu + lam) * J;
    const double den = mu * (1.0 + iJ2) + (1.0 - ::log(J)) * lam * iJ2;
    if (dk_dJ) {
        const double dden = -iJ2 / J * (2.0 * mu + lam + 2.0 * lam * (1.0 - ::log(J)));
        *dk_dJ = st.mobility * ((2.0 * mu + lam) * den - num * dden) / (den * den);
    }
    return st.mobility * num / den;
}

// Particle gather results and derived kinematics.
template <int KIND>
struct PState {
    static const int D = KindTraits<KIND>::D;
    static const int NS = KindTraits<KIND>::NS;
    Shape<D> sh;
    int nid[NS];          // global node id or -1 when outside the grid
    double H[D][D];
    double pbar, pbar_old, pavg_old, pavg, gp[D], dpt, ubar;
};

GW_HD int node_stride(const gw_grid_t &g, int k) {
    return k == 0 ? 1 : (k == 1 ? g.n_grid[0] + 1 : (g.n_grid[0] + 1) * (g.n_grid[1] + 1));
}

// Shape functions and node ids; returns false if a slot with nonzero weight
// falls outside the grid.
template <int KIND>
GW_HD bool particle_shape(const gw_grid_t &g, const double *x, const double *lp, PState<KIND> &s) {
    const int D = KindTraits<KIND>::D, NS = KindTraits<KIND>::NS;
    for (int k = 0; k < D; ++k) gimp_axis(x[k], lp[k], g.h[k], g.inv_h[k], s.sh.ax[k]);
    bool ok = true;
    for (int a = 0; a < NS; ++a) {
        int id = 0;
        bool in = true;
        for (int k = 0; k < D; ++k) {
            int c = s.sh.ax[k].lower + s.sh.idx(a, k);
            if (c < 0 || c > g.n_grid[k]) in = false;
            id += c * node_stride(g, k);
        }
        s.nid[a] = in ? id : -1;
        if (!in && s.sh.W(a) != 0.0) ok = false;
    }
    return ok;
}

template <int KIND>
GW_HD void particle_gather(const double *u_new, const double *u_old, PState<KIND> &s) {
    const int D = KindTraits<KIND>::D, NS = KindTraits<KIND>::NS, NF = KindTraits<KIND>::NF;
    const bool UP = KindTraits<KIND>::UP;
    for (int k = 0; k < D; ++k)
        for (int l = 0; l < D; ++l) s.H[k][l] = 0.0;
    s.pbar = s.pbar_old = s.pavg_old = s.pavg = s.dpt = s.ubar = 0.0;
    for (int k = 0; k < D; ++k) s.gp[k] = 0.0;
    for (int a = 0; a < NS; ++a) {
        const int id = s.nid[a];
        if (id < 0) continue;
        const double W = s.sh.W(a), Wa = s.sh.Wavg(a);
        double G[D];
        for (int k = 0; k < D; ++k) G[k] = s.sh.G(a, k);
        double du[D];
        for (int l = 0; l < D; ++l) du[l] = u_new[(size_t)id * NF + l] - u_old[(size_t)id * NF + l];
        for (int k = 0; k < D; ++k)
            for (int l = 0; l < D; ++l) s.H[k][l] += G[k] * du[l];
        s.ubar += W * du[D - 1];
        if (UP) {
            const double pn = u_new[(size_t)id * NF + D], po = u_old[(size_t)id * NF + D];
            s.pbar += W * pn;
            s.pbar_old += W * po;
            s.pavg += Wa * pn;
            s.pavg_old += Wa * po;
            for (int k = 0; k < D; ++k) s.gp[k] += G[k] * pn;
            s.dpt += (W - Wa) * pn;
        }
    }
}

// ---------------------------------------------------------------- constitutive evaluation
// Everything the residual and the tangent need from one particle.
template <int KIND>
struct PEval {
    static const int D = KindTraits<KIND>::D;
    typedef Layout<KIND> L;
    double Finc[3][3], Finv[D][D];
    double F_new[3][3], b_new[3][3], sigma[3][3];
    double J, J_old;
    double lam, mu;
    double pen;           // penalty residual (0 when the particle is not under the footing)
    double kpen;          // d pen / d ubar
    bool pen_on;
    double pi_new;
    double Q[L::NQ];
    double Dm[L::NQ][L::NT];
};

// Derivative of the isotropic tensor function tau(b) = sum tau_A n_A n_A^T in
// the direction db (symmetric), given the spectral data and d tau_A / d e_B.
// de_B = d lambda_B / (2 lambda_B); coalescing eigenvalues use the limit of
// the divided difference.
GW_HD void spectral_dtau(const double lamb[3], const double V[3][3], const double tauA[3], const double dtau[3][4],
                         const double db[3][3], double devt, double dtau_out[3][3]) {
    // db' = V^T db V
    double T1[3][3], dbp[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) T1[i][j] = db[i][0] * V[0][j] + db[i][1] * V[1][j] + db[i][2] * V[2][j];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) dbp[i][j] = V[0][i] * T1[0][j] + V[1][i] * T1[1][j] + V[2][i] * T1[2][j];
    double de[3];
    for (int B = 0; B < 3; ++B) de[B] = (lamb[B] > 1e-8) ? dbp[B][B] / (2.0 * lamb[B]) : 0.0;
    double dp[3][3];
    for (int A = 0; A < 3; ++A) {
        dp[A][A] = dtau[A][0] * de[0] + dtau[A][1] * de[1] + dtau[A][2] * de[2] + dtau[A][3] * devt;
    }
    for (int A = 0; A < 3; ++A)
        for (int B = 0; B < 3; ++B) {
            if (A == B) continue;
            const double dl = lamb[A] - lamb[B];
            const double sc = fmax(fabs(lamb[A]), fabs(lamb[B]));
            double Dab;
            if (fabs(dl) > 1e-9 * sc) {
                Dab = (tauA[A] - tauA[B]) / dl;
            } else {  // lambda_A -> lambda_B: (d tau_A/d e_A - d tau_A/d e_B) / (2 lambda_A)
                Dab = (dtau[A][A] - dtau[A][B]) / (2.0 * lamb[A]);
            }
            dp[A][B] = Dab * dbp[A][B];
        }
    // dtau = V dp V^T
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) T1[i][j] = V[i][0] * dp[0][j] + V[i][1] * dp[1][j] + V[i][2] * dp[2][j];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) dtau_out[i][j] = T1[i][0] * V[j][0] + T1[i][1] * V[j][1] + T1[i][2] * V[j][2];
}

template <int KIND, bool TANGENT, int MODEL = -1>
GW_HD void particle_eval(const LaunchConst &c, const PState<KIND> &s, const double *xp,
                                              const double *F_old, const double *b_old, double E, double pi_old,
                                              double pi_new_in, double V0, PEval<KIND> &ev) {
    const int D = KindTraits<KIND>::D;
    const bool UP = KindTraits<KIND>::UP;
    typedef Layout<KIND> L;
    const int model = MODEL >= 0 ? MODEL : c.mc.model;
    const double nu = c.nu;
    ev.lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    ev.mu = E / (2.0 * (1.0 + nu));

    double Fo[3][3], bo[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) { Fo[i][j] = F_old[i * 3 + j]; bo[i][j] = b_old[i * 3 + j]; }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) ev.Finc[i][j] = (i == j) ? 1.0 : 0.0;
    for (int i = 0; i < D; ++i)
        for (int j = 0; j < D; ++j) ev.Finc[i][j] += s.H[i][j];
    if (D == 2) {
        const double det = ev.Finc[0][0] * ev.Finc[1][1] - ev.Finc[0][1] * ev.Finc[1][0];
        ev.Finv[0][0] = ev.Finc[1][1] / det;
        ev.Finv[1][1] = ev.Finc[0][0] / det;
        ev.Finv[0][1] = -ev.Finc[0][1] / det;
        ev.Finv[1][0] = -ev.Finc[1][0] / det;
    } else {
        double B3[3][3];
        inv3(ev.Finc, B3);
        for (int i = 0; i < D; ++i)
            for (int j = 0; j < D; ++j) ev.Finv[i][j] = B3[i][j];
    }
    matmul3(ev.Finc, Fo, ev.F_new);
    ev.J = det3(ev.F_new);
    ev.J_old = det3(Fo);
    const double J = ev.J;
    ev.pi_new = pi_new_in;

    // ---------------- stress
    const bool spectral = (model == GW_MODEL_HENCKY || model == GW_MODEL_J2 || model == GW_MODEL_DP ||
                           model == GW_MODEL_NORSAND);
    double lamb[3], V[3][3], tauA[3], dtau[3][4];
    double Mb[3][3];  // b_old Finc^T (for d b_trial)
    if (spectral) {
        double btr[3][3];
        congruence3(ev.Finc, bo, btr);
        eig_sym3(btr, lamb, V);
        double etr[3], e[3];
        for (int A = 0; A < 3; ++A) etr[A] = 0.5 * ::log(fmax(lamb[A], 1e-8));
        const double evt = ::log(J) + c.mc.ns_ev0;
        double pn = ev.pi_new;
        principal_model<double, MODEL>(c.mc, ev.lam, ev.mu, etr, evt, pi_old, pn, tauA, dtau, e, TANGENT);
        ev.pi_new = pn;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double tij = 0.0, bij = 0.0;
                for (int A = 0; A < 3; ++A) {
                    tij += tauA[A] * V[i][A] * V[j][A];
                    bij += ::exp(2.0 * e[A]) * V[i][A] * V[j][A];
                }
                ev.sigma[i][j] = tij / J;
                ev.b_new[i][j] = bij;
            }
        if (TANGENT) {
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) Mb[i][j] = bo[i][0] * ev.Finc[j][0] + bo[i][1] * ev.Finc[j][1] + bo[i][2] * ev.Finc[j][2];
        }
    } else {
        congruence3(ev.Finc, bo, ev.b_new);
        const double lam = ev.lam, mu = ev.mu;
        if (model == GW_MODEL_NEOHOOKEAN) {
            if (D == 2) {  // mpm/mpm_utils.py:915
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) {
                        double FFt = ev.F_new[i][0] * ev.F_new[j][0] + ev.F_new[i][1] * ev.F_new[j][1] + ev.F_new[i][2] * ev.F_new[j][2];
                        ev.sigma[i][j] = mu / J * (FFt - (i == j ? 1.0 : 0.0)) + (i == j ? lam / J * ::log(J) : 0.0);
                    }
            } else {  // PK1 form, mpm/mpm_utils.py:1205-1208
                double Fi[3][3], P[3][3];
                inv3(ev.F_new, Fi);
                const double lnJ = ::log(J);
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) P[i][j] = mu * (ev.F_new[i][j] - Fi[j][i]) + lam * lnJ * Fi[j][i];
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j)
                        ev.sigma[i][j] = 1.0 / J * (P[i][0] * ev.F_new[j][0] + P[i][1] * ev.F_new[j][1] + P[i][2] * ev.F_new[j][2]);
            }
        } else {  // small-strain linear elasticity on sym(F) - I
            double eps[3][3];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) eps[i][j] = 0.5 * (ev.F_new[i][j] + ev.F_new[j][i]) - (i == j ? 1.0 : 0.0);
            const double tr = eps[0][0] + eps[1][1] + eps[2][2];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) ev.sigma[i][j] = (i == j ? lam * tr : 0.0) + 2.0 * mu * eps[i][j];
        }
    }

    // ---------------- penalty footing
    ev.pen = 0.0;
    ev.kpen = 0.0;
    ev.pen_on = false;
    if (c.st.has_footing) {
        const int v = D - 1;
        const double height = c.st.footing_initial_height + (c.st.current_step + 1.0) * c.st.footing_incr_disp;
        bool sel = xp[v] >= height && xp[0] > c.st.footing_min[0] && xp[0] < c.st.footing_max[0];
        if (D == 3) sel = sel && xp[1] > c.st.footing_min[1] && xp[1] < c.st.footing_max[1];
        if (sel) {
            const double area = (D == 2) ? c.g.h[0] / c.st.PPD : (c.g.h[0] / c.st.PPD) * (c.g.h[1] / c.st.PPD);
            ev.kpen = E * c.st.penalty_factor * area;
            const double penetration = height - (xp[v] + s.ubar);
            ev.pen = -penetration * ev.kpen;
            if (c.st.footing_stable) {  // attractive spring (extension)
                ev.pen = -ev.pen;
                ev.kpen = -ev.kpen;
            }
            ev.pen_on = true;
        }
    }

    // ---------------- Q values
    const double pb = UP ? s.pbar : 0.0;
    for (int i = 0; i < D; ++i)
        for (int j = 0; j < D; ++j) {
            double a = 0.0;
            for (int k = 0; k < D; ++k) a += ev.Finv[k][i] * (ev.sigma[k][j] - (k == j ? pb : 0.0));
            ev.Q[L::QU + i * D + j] = V0 * J * a;
        }
    const double phi_s0 = 1.0 - c.st.phi_initial;
    if (UP) {
        const double nfl = 1.0 - phi_s0 / J;
        const double rho_mix = nfl * 1.0 + (1.0 - nfl) * c.st.p_rho;
        ev.Q[L::QS] = rho_mix * V0 * J;
    } else {
        ev.Q[L::QS] = c.st.p_rho / J * (V0 * J);
    }
    ev.Q[L::QPEN] = ev.pen;
    double FtFg[D];  // mass-balance flux direction before the V0 J dt mob factor
    const double tau_ppp = 0.5 / ev.mu;
    if (UP) {
        ev.Q[L::QM1] = V0 * J * (::log(J) - ::log(ev.J_old));
        double gsp[D];  // grad p: 2D spatial (Finv gp), 3D reference gradient (mpm_utils.py:950, 1194)
        for (int k = 0; k < D; ++k) {
            if (D == 2) {
                gsp[k] = 0.0;
                for (int l = 0; l < D; ++l) gsp[k] += ev.Finv[k][l] * s.gp[l];
            } else {
                gsp[k] = s.gp[k];
            }
        }
        for (int i = 0; i < D; ++i) {
            FtFg[i] = 0.0;
            for (int k = 0; k < D; ++k) FtFg[i] += ev.Finv[k][i] * gsp[k];
            ev.Q[L::QM2 + i] = V0 * J * c.st.dt * mobility_of(c.st, J, ev.lam, ev.mu, nullptr) * FtFg[i];
        }
        const double cold = s.pbar_old - s.pavg_old;
        ev.Q[L::QM3] = V0 * J * tau_ppp * (s.dpt - cold);
    }

    if (!TANGENT) return;

    // ---------------- dQ/dtheta
    for (int q = 0; q < L::NQ; ++q)
        for (int t = 0; t < L::NT; ++t) ev.Dm[q][t] = 0.0;
    for (int k = 0; k < D; ++k)
        for (int l = 0; l < D; ++l) {
            const int t = L::TH + k * D + l;
            // dFinc = E_kl ; dFinv = -Finv E_kl Finv ; dJ = J Finv_lk
            double dFinv[D][D];
            for (int i = 0; i < D; ++i)
                for (int j = 0; j < D; ++j) dFinv[i][j] = -ev.Finv[i][k] * ev.Finv[l][j];
            const double dJ = J * ev.Finv[l][k];
            double dsig[3][3];
            if (spectral) {
                double db[3][3];
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) db[i][j] = (i == k ? Mb[l][j] : 0.0) + (j == k ? Mb[l][i] : 0.0);
                double dtau_m[3][3];
                spectral_dtau(lamb, V, tauA, dtau, db, dJ / J, dtau_m);
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) dsig[i][j] = dtau_m[i][j] / J - ev.sigma[i][j] * dJ / J;
            } else if (model == GW_MODEL_NEOHOOKEAN) {
                // d(J sigma) = mu (dF F^T + F dF^T) + lam dJ/J I ;  dF = E_kl F_old (row k)
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) {
                        double dFFt = 0.0;
                        for (int m = 0; m < 3; ++m) {
                            const double dFim = (i == k) ? Fo[l][m] : 0.0;
                            const double dFjm = (j == k) ? Fo[l][m] : 0.0;
                            dFFt += dFim * ev.F_new[j][m] + ev.F_new[i][m] * dFjm;
                        }
                        const double dJs = ev.mu * dFFt + (i == j ? ev.lam * dJ / J : 0.0);
                        dsig[i][j] = dJs / J - ev.sigma[i][j] * dJ / J;
                    }
            } else {
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) {
                        const double dFij = (i == k) ? Fo[l][j] : 0.0;
                        const double dFji = (j == k) ? Fo[l][i] : 0.0;
                        dsig[i][j] = 2.0 * ev.mu * 0.5 * (dFij + dFji);
                    }
                double dtr = 0.0;
                for (int i = 0; i < 3; ++i) dtr += (i == k) ? Fo[l][i] : 0.0;
                for (int i = 0; i < 3; ++i) dsig[i][i] += ev.lam * dtr;
            }
            // Qu = V0 J Finv^T (sigma - pbar I)
            for (int i = 0; i < D; ++i)
                for (int j = 0; j < D; ++j) {
                    double a = 0.0, da = 0.0, dd = 0.0;
                    for (int m = 0; m < D; ++m) {
                        const double sm = ev.sigma[m][j] - (m == j ? pb : 0.0);
                        a += ev.Finv[m][i] * sm;
                        da += dFinv[m][i] * sm;
                        dd += ev.Finv[m][i] * dsig[m][j];
                    }
                    ev.Dm[L::QU + i * D + j][t] = V0 * (dJ * a + J * da + J * dd);
                }
            if (UP) {
                ev.Dm[L::QS][t] = V0 * dJ;
                ev.Dm[L::QM1][t] = V0 * dJ * (::log(J) - ::log(ev.J_old) + 1.0);
                double dmob = 0.0;
                const double mob = mobility_of(c.st, J, ev.lam, ev.mu, &dmob);
                const double fac = V0 * c.st.dt;
                for (int i = 0; i < D; ++i) {
                    double dF = 0.0;
                    if (D == 2) {
                        // FtFg = Finv^T Finv gp
                        double g1[D], dg1[D];
                        for (int m = 0; m < D; ++m) {
                            g1[m] = 0.0; dg1[m] = 0.0;
                            for (int n = 0; n < D; ++n) { g1[m] += ev.Finv[m][n] * s.gp[n]; dg1[m] += dFinv[m][n] * s.gp[n]; }
                        }
                        for (int m = 0; m < D; ++m) dF += dFinv[m][i] * g1[m] + ev.Finv[m][i] * dg1[m];
                    } else {
                        for (int m = 0; m < D; ++m) dF += dFinv[m][i] * s.gp[m];
                    }
                    ev.Dm[L::QM2 + i][t] = fac * (dJ * (mob + J * dmob) * FtFg[i] + J * mob * dF);
                }
                ev.Dm[L::QM3][t] = V0 * dJ * tau_ppp * (s.dpt - (s.pbar_old - s.pavg_old));
            }
        }
    // ubar lane
    ev.Dm[L::QPEN][L::TU] = ev.pen_on ? ev.kpen : 0.0;
    if (UP) {
        // pbar lane: Qu -= V0 J Finv^T pbar I
        for (int i = 0; i < D; ++i)
            for (int j = 0; j < D; ++j) ev.Dm[L::QU + i * D + j][L::TP] = -V0 * J * ev.Finv[j][i];
        // grad~p lanes
        const double fac = V0 * J * c.st.dt * mobility_of(c.st, J, ev.lam, ev.mu, nullptr);
        for (int i = 0; i < D; ++i)
            for (int k = 0; k < D; ++k) {
                double v;
                if (D == 2) {
                    v = 0.0;  // (Finv^T Finv)_ik
                    for (int m = 0; m < D; ++m) v += ev.Finv[m][i] * ev.Finv[m][k];
                } else {
                    v = ev.Finv[k][i];
                }
                ev.Dm[L::QM2 + i][L::TG + k] = fac * v;
            }
        ev.Dm[L::QM3][L::TD] = V0 * J * tau_ppp;
    }
}

// Residual row values of slot a (nf entries), literal reference formulas.
template <int KIND>
GW_HD void residual_rows(const LaunchConst &c, const PState<KIND> &s, const PEval<KIND> &ev,
                                              int a, const double *fext, const double *ftr, double V0, double *r) {
    const int D = KindTraits<KIND>::D;
    const bool UP = KindTraits<KIND>::UP;
    const double W = s.sh.W(a);
    double G[D], wg[D];
    for (int k = 0; k < D; ++k) G[k] = s.sh.G(a, k);
    for (int i = 0; i < D; ++i) {
        wg[i] = 0.0;
        for (int k = 0; k < D; ++k) wg[i] += ev.Finv[i][k] * G[k];
    }
    const double Vn = V0 * ev.J;
    const double ramp = (c.st.current_step + 1.0) / c.st.total_steps;
    const double gv = -c.st.gravity_mag * (c.st.gravity_full ? 1.0 : ramp);
    const double pb = UP ? s.pbar : 0.0;
    double rho;
    if (UP) {
        const double nfl = 1.0 - (1.0 - c.st.phi_initial) / ev.J;
        rho = nfl * 1.0 + (1.0 - nfl) * c.st.p_rho;
    } else {
        rho = c.st.p_rho / ev.J;
    }
    for (int j = 0; j < D; ++j) {
        double a1 = 0.0;
        for (int i = 0; i < D; ++i) a1 += wg[i] * (ev.sigma[i][j] - (i == j ? pb : 0.0));
        const double gj = (j == D - 1) ? gv : 0.0;
        double v = (-a1 + W * rho * gj) * Vn;
        if (KIND != GW_KIND_COUPLED3D) v += W * fext[j];
        if (KIND == GW_KIND_COUPLED2D) v += W * ftr[j];
        if (j == D - 1 && ev.pen_on) v += ev.pen * W;
        r[j] = v;
    }
    if (UP) {
        const double Wa = s.sh.Wavg(a);
        double gsp[D];
        for (int k = 0; k < D; ++k) {
            if (D == 2) {
                gsp[k] = 0.0;
                for (int l = 0; l < D; ++l) gsp[k] += ev.Finv[k][l] * s.gp[l];
            } else {
                gsp[k] = s.gp[k];
            }
        }
        double dot = 0.0;
        const double mob = mobility_of(c.st, ev.J, ev.lam, ev.mu, nullptr);
        for (int k = 0; k < D; ++k) dot += wg[k] * (mob * gsp[k]);
        double rm = (W * (::log(ev.J) - ::log(ev.J_old)) + dot * c.st.dt) * Vn;
        const double tau_ppp = 0.5 / ev.mu;
        rm += (tau_ppp * (W - Wa) * (s.pbar - s.pavg - (s.pbar_old - s.pavg_old))) * Vn;
        r[D] = rm;
    }
}

}  // namespace
}  // namespace gw
