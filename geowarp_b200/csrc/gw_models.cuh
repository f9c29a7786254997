// Constitutive models in principal logarithmic-strain space, one particle per
// thread, templated on the scalar (double, float or Dual<4, .> to obtain the
// algorithmic tangent through the fixed-count local iterations).
//
//   Hencky elasticity  mpm/mpm_utils.py:537-542
//   J2 radial return   materials/plasticity.py:8-37
//   Drucker-Prager     problems/material_tests/triaxial_DruckerPrager.py:119-412
//   NorSand            problems/material_tests/triaxial_NorSand.py:155-400
#pragma once
#include "gw_math.cuh"
#include "../../include/geowarp_b200.h"

namespace gw {
namespace {  // internal linkage: each translation unit compiles the kernels it launches

// Per-material constants, precomputed on the host side of each launch.
struct MatConst {
    int model;
    int dp_cutoff;                 // DP: skip the return when P_trial >= 0 (reference behaviour)
    double kappa;                  // J2
    double A_phi, B_phi, A_psi, B_psi, sf;  // DP (triaxial_DruckerPrager.py:130-134, 151-155)
    double ns_kappa, ns_tl, ns_M, ns_N, ns_beta, ns_vc0, ns_p0, ns_v0, ns_h, ns_mu, ns_ev0;
    double tip_tangent;            // DP: Jacobian-only elastic fraction at the cone tip
};

inline MatConst make_matconst(const gw_material_t &m) {
    MatConst c{};
    c.model = m.model;
    c.dp_cutoff = m.dp_tension_cutoff;
    c.kappa = m.kappa;
    const double pi_ref = 3.14159265358979;  // constant hard-coded by the reference
    double cp = ::cos(m.friction_angle * pi_ref / 180.0), sp = ::sin(m.friction_angle * pi_ref / 180.0);
    double cd = ::cos(m.dilation_angle * pi_ref / 180.0), sd = ::sin(m.dilation_angle * pi_ref / 180.0);
    c.A_phi = 2.0 * ::sqrt(6.0) * m.cohesion * cp / (3.0 - sp);
    c.B_phi = 2.0 * ::sqrt(6.0) * sp / (3.0 - sp);
    c.A_psi = 2.0 * ::sqrt(6.0) * m.cohesion * cd / (3.0 - sd);
    c.B_psi = 2.0 * ::sqrt(6.0) * sd / (3.0 - sd);
    c.sf = m.shape_factor;
    c.ns_kappa = m.ns_kappa; c.ns_tl = m.ns_tilde_lambda; c.ns_M = m.ns_M; c.ns_N = m.ns_N;
    c.ns_beta = m.ns_beta; c.ns_vc0 = m.ns_vc0; c.ns_p0 = m.ns_p0; c.ns_v0 = m.ns_v0; c.ns_h = m.ns_h;
    c.ns_mu = m.ns_shear_modulus; c.ns_ev0 = m.ns_eps_v0;
    c.tip_tangent = m.dp_tip_tangent;
    return c;
}

template <typename T, typename LT>
GW_HD void tau_hencky(const T e[3], LT lam, LT mu, T tau[3]) {
    T tr = e[0] + e[1] + e[2];
#pragma unroll
    for (int i = 0; i < 3; ++i) tau[i] = lam * tr + 2.0 * mu * e[i];
}

// ------------------------------------------------------------------ J2
template <typename T, typename R, typename LT>
GW_HD void rm_j2(const T etr[3], LT lam, LT mu, R kappa, T e[3]) {
    T tau[3];
    tau_hencky(etr, lam, mu, tau);
    T P = (tau[0] + tau[1] + tau[2]) / R(3);
    T S[3] = {tau[0] - P, tau[1] - P, tau[2] - P};
    T nrm = gsqrt(S[0] * S[0] + S[1] * S[1] + S[2] * S[2]);
    if (val(nrm) > kappa) {
        T dl = (nrm - kappa) / (2.0 * mu);
#pragma unroll
        for (int i = 0; i < 3; ++i) e[i] = etr[i] - dl * (S[i] / nrm);
    } else {
#pragma unroll
        for (int i = 0; i < 3; ++i) e[i] = etr[i];
    }
}

// ------------------------------------------------------------------ Drucker-Prager
template <typename T, typename R>
GW_HD T dp_yield(const T &P, const T &Q, R A, R B, R sf) {
    T om = R(2) / R(3) * Q * Q + sf * sf * A * A;
    return gsqrt(om) - (A - B * P);
}

// gradient of the yield function (A_phi,B_phi) or plastic potential (A_psi,B_psi)
template <typename T, typename R>
GW_HD void dp_grad(const T tau[3], const T &Q, R A, R B, R sf, T g[3]) {
    T om = R(2) / R(3) * Q * Q + sf * sf * A * A;
    T dFdQ = R(2) / R(3) * Q / gsqrt(om);
    T Qt = Q;
    R sgn = val(Q) < R(0) ? R(-1) : R(1);
    if (fabs(val(Q)) < R(1e-10)) Qt = T(R(1e-10) * sgn);
    T gq0 = R(0.5) / Qt * (R(2) * tau[0] - tau[1] - tau[2]);
    T gq1 = R(0.5) / Qt * (R(2) * tau[1] - tau[0] - tau[2]);
    T gq2 = R(0.5) / Qt * (R(2) * tau[2] - tau[0] - tau[1]);
    g[0] = B / R(3) + dFdQ * gq0;
    g[1] = B / R(3) + dFdQ * gq1;
    g[2] = B / R(3) + dFdQ * gq2;
}

template <typename T, typename R>
GW_HD void dp_hess(const T S[3], const T &Q, R A, R sf, T H[3][3]) {
    T chi = gsqrt(S[0] * S[0] + S[1] * S[1] + S[2] * S[2]);
    if (fabs(val(chi)) < R(1e-10)) chi = T(R(1e-10));
    T c1 = R(1.224744871391589) / chi;  // gsqrt(3/2)
    T chi2 = chi * chi;
    T gQ[3] = {c1 * S[0], c1 * S[1], c1 * S[2]};
    T om = R(2) / R(3) * Q * Q + sf * sf * A * A;
    T som = gsqrt(om);
    T dFdQ = R(2) / R(3) * Q / som;
    T d2 = R(2) / R(3) / som - R(4) / R(9) * Q * Q / (om * som);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            T hq = c1 * ((i == j ? R(1) : R(0)) - R(1) / R(3) - S[i] * S[j] / chi2);
            H[i][j] = dFdQ * hq + d2 * gQ[i] * gQ[j];
        }
}

template <typename T, typename R, typename LT>
GW_HD void dp_invariants(const T e[3], LT lam, LT mu, T tau[3], T &P, T S[3], T &Q) {
    tau_hencky(e, lam, mu, tau);
    P = (tau[0] + tau[1] + tau[2]) / R(3);
#pragma unroll
    for (int i = 0; i < 3; ++i) S[i] = tau[i] - P;
    Q = gsqrt(S[0] * S[0] + S[1] * S[1] + S[2] * S[2]) * R(1.224744871391589);
}

template <typename T, typename R, typename LT>
GW_HD void rm_dp(const T etr[3], LT lam, LT mu, const MatConst &c, T e[3]) {
    const R Af = R(c.A_phi), Bf = R(c.B_phi), Ap = R(c.A_psi), Bp = R(c.B_psi), sf = R(c.sf);
    T tau[3], P, S[3], Q;
    dp_invariants<T, R, LT>(etr, lam, mu, tau, P, S, Q);
#pragma unroll
    for (int i = 0; i < 3; ++i) e[i] = etr[i];
    T y0 = dp_yield(P, Q, Af, Bf, sf);
    if (val(y0) < R(1e-10)) return;     // elastic
    if (c.dp_cutoff && val(P) >= R(0)) return;  // apex return not implemented in the reference (:347-349)
    if (!c.dp_cutoff && Bf > R(0)) {
        // extension: at or beyond the tip P_tip = A (1 - sf) / B no cone state is
        // reachable; return to the tip (isotropic state), continuous with the cone return
        const R p_tip = Af * (R(1) - sf) / Bf;
        if (val(P) >= p_tip) {
            const LT K3 = (lam + 2.0 * mu / 3.0) * 3.0;
            // the tip state is fixed (zero exact tangent); a nonzero tip_tangent keeps
            // that fraction of the trial strain's derivative, value unchanged
            const R frac = R(c.tip_tangent);
#pragma unroll
            for (int i = 0; i < 3; ++i) e[i] = T(R(0)) + p_tip / K3 + frac * (etr[i] - val(etr[i]));
            return;
        }
    }
    T dl = T(R(0));
    const LT a_d = lam + 2.0 * mu, a_o = lam;  // elastic_a = lam 1 1^T + 2 mu I
    for (int it = 0; it < 10; ++it) {
        T gg[3], gf[3], hg[3][3];
        dp_grad(tau, Q, Ap, Bp, sf, gg);
        dp_grad(tau, Q, Af, Bf, sf, gf);
        dp_hess(S, Q, Ap, sf, hg);
        T y = dp_yield(P, Q, Af, Bf, sf);
        T M[4][4], rhs[4], x[4];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            rhs[i] = e[i] - etr[i] + dl * gg[i];
            // (hess_g @ a)_ij = sum_k hg_ik a_kj ;  grad_f_eps_j = sum_i gf_i a_ij
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                T hge = hg[i][0] * (j == 0 ? a_d : a_o) + hg[i][1] * (j == 1 ? a_d : a_o) + hg[i][2] * (j == 2 ? a_d : a_o);
                M[i][j] = (i == j ? T(R(1)) : T(R(0))) + dl * hge;
            }
            M[i][3] = gg[i];
        }
#pragma unroll
        for (int j = 0; j < 3; ++j)
            M[3][j] = gf[0] * (j == 0 ? a_d : a_o) + gf[1] * (j == 1 ? a_d : a_o) + gf[2] * (j == 2 ? a_d : a_o);
        M[3][3] = T(R(0));
        rhs[3] = y;
        solve4(M, rhs, x);
#pragma unroll
        for (int i = 0; i < 3; ++i) e[i] = e[i] - x[i];
        dl = dl - x[3];
        dp_invariants<T, R, LT>(e, lam, mu, tau, P, S, Q);
    }
}

// ------------------------------------------------------------------ NorSand
template <typename T, typename R>
GW_HD T ns_eta(R M, R N, const T &P, const T &pi) {
    if (fabs(N) < R(1e-10)) return M * (R(1) + glog(pi / P));
    return (M / N) * (R(1) - (R(1) - N) * gpow(P / pi, N / (R(1) - N)));
}
template <typename T, typename R>
GW_HD T ns_dEtadP(R M, R N, const T &P, const T &pi) {
    if (fabs(N) < R(1e-10)) return M * R(-1) / P;
    return M * (R(-1) * gpow(P / pi, (R(2) * N - R(1)) / (R(1) - N)) / pi);
}
template <typename T, typename R>
GW_HD T ns_dEtadPi(R M, R N, const T &P, const T &pi) {
    if (fabs(N) < R(1e-10)) return M / pi;
    return M * (R(-1) * gpow(P / pi, (R(2) * N - R(1)) / (R(1) - N)) * (-P) / (pi * pi));
}
template <typename T, typename R>
GW_HD T ns_eps_s(const T e[3]) {
    return gsqrt(R(2) / R(9) * ((e[0] - e[1]) * (e[0] - e[1]) + (e[1] - e[2]) * (e[1] - e[2]) + (e[0] - e[2]) * (e[0] - e[2])));
}

// Returns true when the point was plastic (pi_new written).
template <typename T, typename R>
GW_HD bool rm_norsand(const T etr[3], const T &eps_v_total, R pi_old, const MatConst &c, T e[3], R &pi_new) {
    const R kap = R(c.ns_kappa), tl = R(c.ns_tl), M = R(c.ns_M), N = R(c.ns_N), beta = R(c.ns_beta);
    const R vc0 = R(c.ns_vc0), p0 = R(c.ns_p0), v0 = R(c.ns_v0), h = R(c.ns_h), mu = R(c.ns_mu), ev0 = R(c.ns_ev0);
    const R tol = R(1e-10);
    const R ab = R(-3.5) / beta;
    T eps_v = etr[0] + etr[1] + etr[2];
    T eps_s = ns_eps_s<T, R>(etr);
    T nd[3];
    if (val(eps_s) > tol) {
#pragma unroll
        for (int i = 0; i < 3; ++i) nd[i] = R(0.816496580927726) * (etr[i] - eps_v / R(3)) / eps_s;  // gsqrt(2/3)
    } else {
#pragma unroll
        for (int i = 0; i < 3; ++i) nd[i] = T(R(0));
    }
    T P = p0 * gexp(-(eps_v - ev0) / kap);
    T Q = R(3) * mu * eps_s;
    T new_v = gexp(eps_v_total) * v0;
#pragma unroll
    for (int i = 0; i < 3; ++i) e[i] = etr[i];
    if (val(eps_v) > tol) {  // tension: zero strain (triaxial_NorSand.py:295-296)
#pragma unroll
        for (int i = 0; i < 3; ++i) e[i] = T(R(0));
        return false;
    }
    T y0 = Q + ns_eta(M, N, P, T(pi_old)) * P;
    if (val(y0) < tol) return false;
    T pi = T(pi_old), dl = T(R(0));
    for (int it = 0; it < 15; ++it) {
        T ev = e[0] + e[1] + e[2];
        T es = ns_eps_s<T, R>(e);
        T dEdP = ns_dEtadP(M, N, P, pi);
        T dEdPi = ns_dEtadPi(M, N, P, pi);
        T eta = ns_eta(M, N, P, pi);
        T dFdP = (eta - M) / (R(1) - N);
        const R dFdQ = R(1);
        T psi_i = new_v - vc0 + tl * glog(-pi);
        T base = R(1) - ab * psi_i * N / M;
        T pistar = (fabs(N) < tol) ? P * gexp(ab * psi_i / M) : P * gpow(base, (N - R(1)) / N);
        T y = Q + eta * P;
        T hard = pi - pi_old + h * (pi - pistar) * dl;
        T omn = -(ev - ev0) / kap;
        T dPde = p0 * gexp(omn) / (-kap);
        T d2F_dPdepsv = R(1) / (R(1) - N) * dEdP * dPde;
        T d2F_dPdPi = R(1) / (R(1) - N) * dEdPi;
        T dFdepsv = (dEdP * P + eta) * dPde;
        const R dFdepss = R(3) * mu;
        T dFdPi = P * dEdPi;
        T dPs_dP = (fabs(N) < R(1e-10)) ? gexp(ab * psi_i / M) : gpow(base, (N - R(1)) / N);
        T dPsii_dPi = tl / pi;
        T dPs_dPi = (fabs(N) < R(1e-10)) ? P * gexp(ab * psi_i / M) * ab / M * dPsii_dPi
                                          : P * (N - R(1)) / N * gpow(R(1) / base, R(1) / N) * (-ab * N / M) * dPsii_dPi;
        T dHdepsv = -h * dl * dPs_dP * dPde;
        T dHdPi = R(1) + h * dl * (R(1) - dPs_dPi);
        T Mx[4][4], rhs[4], x[4];
        rhs[0] = ev - eps_v + dl * beta * dFdP;
        rhs[1] = es - eps_s + dl * dFdQ;
        rhs[2] = y;
        rhs[3] = hard;
        Mx[0][0] = R(1) + dl * beta * d2F_dPdepsv; Mx[0][1] = T(R(0)); Mx[0][2] = beta * dFdP; Mx[0][3] = dl * beta * d2F_dPdPi;
        Mx[1][0] = T(R(0)); Mx[1][1] = T(R(1)); Mx[1][2] = T(dFdQ); Mx[1][3] = T(R(0));
        Mx[2][0] = dFdepsv; Mx[2][1] = T(dFdepss); Mx[2][2] = T(R(0)); Mx[2][3] = dFdPi;
        Mx[3][0] = dHdepsv; Mx[3][1] = T(R(0)); Mx[3][2] = h * (pi - pistar); Mx[3][3] = dHdPi;
        solve4(Mx, rhs, x);
        T nev = ev - x[0];
        T nes = es - x[1];
        dl = dl - x[2];
        pi = pi - x[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) e[i] = nev / R(3) + nes * nd[i] * R(1.224744871391589);
        T tr = e[0] + e[1] + e[2];
        P = p0 * gexp(-(tr - ev0) / kap);
        Q = R(3) * mu * ns_eps_s<T, R>(e);
    }
    pi_new = val(pi);
    return true;
}

template <typename T, typename R>
GW_HD void tau_norsand(const T e[3], const MatConst &c, T tau[3]) {
    T tr = e[0] + e[1] + e[2];
    T om = -(tr - R(c.ns_ev0)) / R(c.ns_kappa);
    T pp = -R(c.ns_p0) * R(c.ns_kappa) * gexp(om) / (-R(c.ns_kappa));
#pragma unroll
    for (int i = 0; i < 3; ++i) tau[i] = pp + R(2) / R(3) * R(c.ns_mu) * (R(3) * e[i] - tr);
}

// ------------------------------------------------------------------ dispatcher
// Principal model with its algorithmic tangent: lanes 0..2 seed e_trial_B,
// lane 3 seeds the total volumetric strain (NorSand's specific volume).
// Outputs tau[A], dtau[A][lane], e_out[A]; pi_new updated for plastic NorSand.
// MODEL (GW_MODEL_*) fixed at compile time drops the other models' code from
// the caller's instantiation; MODEL < 0 dispatches on c.model at run time.
template <typename R, int MODEL = -1>
GW_HD void principal_model(const MatConst &c, R lam, R mu, const R etr_v[3], R eps_v_total, R pi_old, R &pi_new,
                           R tau_v[3], R dtau[3][4], R e_out[3], bool want_tangent, R (*de)[4] = nullptr) {
    typedef Dual<4, R> T;
    T etr[3], e[3], tau[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        etr[i] = T(etr_v[i]);
        if (want_tangent) etr[i].d[i] = R(1);
    }
    T evt = T(eps_v_total);
    if (want_tangent) evt.d[3] = R(1);
    switch (MODEL >= 0 ? MODEL : c.model) {
        case GW_MODEL_J2:
            rm_j2<T, R, R>(etr, lam, mu, R(c.kappa), e);
            tau_hencky(e, lam, mu, tau);
            break;
        case GW_MODEL_DP:
            rm_dp<T, R, R>(etr, lam, mu, c, e);
            tau_hencky(e, lam, mu, tau);
            break;
        case GW_MODEL_NORSAND: {
            R pn = pi_new;
            if (rm_norsand(etr, evt, pi_old, c, e, pn)) pi_new = pn;
            tau_norsand<T, R>(e, c, tau);
            break;
        }
        default:  // Hencky elasticity
#pragma unroll
            for (int i = 0; i < 3; ++i) e[i] = etr[i];
            tau_hencky(e, lam, mu, tau);
            break;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        tau_v[i] = tau[i].v;
        e_out[i] = e[i].v;
#pragma unroll
        for (int l = 0; l < 4; ++l) dtau[i][l] = tau[i].d[l];
        if (de)
#pragma unroll
            for (int l = 0; l < 4; ++l) de[i][l] = e[i].d[l];
    }
}

}  // namespace
}  // namespace gw
