"""Constitutive models in principal logarithmic-strain space (oracle).

Every return map takes the trial elastic log strains e_trial[N, 3] (principal
values) and returns the corrected strains.  Arrays may be complex so that
complex-step derivatives propagate through the fixed local iteration counts,
which is what Warp's tape differentiates in the reference.

  * Hencky elasticity   mpm/mpm_utils.py:537-542
  * J2 radial return    materials/plasticity.py:8-37
  * Drucker-Prager      problems/material_tests/triaxial_DruckerPrager.py:119-412
  * NorSand             problems/material_tests/triaxial_NorSand.py:155-400
"""
import numpy as np

PI_REF = 3.14159265358979  # the constant the reference hard-codes (triaxial_DruckerPrager.py:128)


def kirchhoff_hencky(e, lam, mu):
    """tau_A = lambda tr(e) + 2 mu e_A (mpm/mpm_utils.py:541-542)."""
    tr = e.sum(1, keepdims=True)
    return lam * tr + 2.0 * mu * e


def return_map_j2(e_tr, lam, mu, kappa):
    """Radial return of materials/plasticity.py:8-37."""
    tau = kirchhoff_hencky(e_tr, lam, mu)
    P = tau.sum(1, keepdims=True) / 3.0
    S = tau - P
    nrm = np.sqrt(S[:, 0] ** 2 + S[:, 1] ** 2 + S[:, 2] ** 2)[:, None]
    plastic = np.real(nrm) > kappa
    with np.errstate(divide="ignore", invalid="ignore"):
        dlam = (nrm - kappa) / (2.0 * mu)
        e_pl = e_tr - dlam * S / nrm
    return np.where(plastic, e_pl, e_tr)


# ---------------------------------------------------------------- Drucker-Prager
def _dp_AB(angle_deg, cohesion):
    c = np.cos(angle_deg * PI_REF / 180.0)
    s = np.sin(angle_deg * PI_REF / 180.0)
    A = 2.0 * np.sqrt(6.0) * cohesion * c / (3.0 - s)
    B = 2.0 * np.sqrt(6.0) * s / (3.0 - s)
    return A, B


def dp_yield(P, Q, phi, c, sf):
    """triaxial_DruckerPrager.py:120-138."""
    A, B = _dp_AB(phi, c)
    om = 2.0 / 3.0 * Q * Q + sf * sf * A * A
    return np.sqrt(om) - (A - B * P)


def _dp_grad(tau, Q, angle, c, sf):
    """triaxial_DruckerPrager.py:140-226 (potential and yield gradients share it)."""
    A, B = _dp_AB(angle, c)
    om = 2.0 / 3.0 * Q * Q + sf * sf * A * A
    dFdP = B
    dFdQ = 2.0 / 3.0 * Q / np.sqrt(om)
    sgn = np.where(np.real(Q) < 0, -1.0, 1.0)
    small = np.abs(np.real(Q)) < 1e-10
    Qt = np.where(small, 1e-10 * sgn, Q)
    t0, t1, t2 = tau[:, 0], tau[:, 1], tau[:, 2]
    gQ = np.stack([0.5 / Qt * (2 * t0 - t1 - t2),
                   0.5 / Qt * (2 * t1 - t0 - t2),
                   0.5 / Qt * (2 * t2 - t0 - t1)], 1)
    return dFdP / 3.0 + dFdQ[:, None] * gQ


def _dp_hess(S, Q, psi, c, sf):
    """triaxial_DruckerPrager.py:240-282."""
    trS2 = S[:, 0] ** 2 + S[:, 1] ** 2 + S[:, 2] ** 2
    chi = np.sqrt(trS2)
    chi = np.where(np.abs(np.real(chi)) < 1e-10, 1e-10, chi)
    c1 = np.sqrt(1.5) / chi
    gQ = c1[:, None] * S
    eye = np.eye(3)
    hQ = c1[:, None, None] * (eye[None] - 1.0 / 3.0 - S[:, :, None] * S[:, None, :] / (chi * chi)[:, None, None])
    A, B = _dp_AB(psi, c)
    om = 2.0 / 3.0 * Q * Q + sf * sf * A * A
    dFdQ = 2.0 / 3.0 * Q / np.sqrt(om)
    d2 = 2.0 / 3.0 / np.sqrt(om) - 4.0 / 9.0 * Q * Q / (om * np.sqrt(om))
    return dFdQ[:, None, None] * hQ + d2[:, None, None] * gQ[:, :, None] * gQ[:, None, :]


def return_map_dp(e_tr, lam, mu, phi, psi, c, sf, n_local=10, tension_cutoff=True):
    """Drucker-Prager return map, fixed n_local local Newton iterations.

    Follows return_mapping_DruckerPrager, triaxial_DruckerPrager.py:308-412:
    elastic if f < 1e-10, trial state kept when P_trial >= 0 (apex return not
    implemented in the reference), else a 4x4 Newton in (e_1, e_2, e_3, dlambda).
    tension_cutoff=False replaces the P_trial >= 0 guard by a continuous
    completion (extension): the cone return for P_trial below the tip of the
    yield surface, P_tip = A (1 - sf) / B, and a return to the tip (isotropic
    state at P_tip) at or beyond it, where the cone return with this flow rule
    has no solution.
    """
    n = e_tr.shape[0]
    lam_v = np.broadcast_to(np.asarray(lam, dtype=np.float64).reshape(-1, 1), (n, 1))
    mu_v = np.broadcast_to(np.asarray(mu, dtype=np.float64).reshape(-1, 1), (n, 1))
    a = lam_v[:, :, None] * np.ones((3, 3)) + 2.0 * mu_v[:, :, None] * np.eye(3)

    def inv(e):
        tau = kirchhoff_hencky(e, lam, mu)
        P = tau.sum(1) / 3.0
        S = tau - P[:, None]
        Q = np.sqrt(S[:, 0] ** 2 + S[:, 1] ** 2 + S[:, 2] ** 2) * np.sqrt(1.5)
        return tau, P, S, Q

    tau, P, S, Q = inv(e_tr)
    y0 = dp_yield(P, Q, phi, c, sf)
    elastic = (np.real(y0) < 1e-10) | ((np.real(P) >= 0.0) & tension_cutoff)
    A_f, B_f = _dp_AB(phi, c)
    p_tip = A_f * (1.0 - sf) / B_f if B_f > 0 else np.inf
    apex = (~elastic) & (not tension_cutoff) & (np.real(P) >= p_tip)
    e = e_tr.copy()
    dl = np.zeros(e_tr.shape[0], dtype=e_tr.dtype)
    eye3 = np.eye(3)
    for _ in range(n_local):
        gg = _dp_grad(tau, Q, psi, c, sf)
        gf = _dp_grad(tau, Q, phi, c, sf)
        gfe = np.einsum("ni,nij->nj", gf, a)
        hg = _dp_hess(S, Q, psi, c, sf)
        hge = np.einsum("nij,njk->nik", hg, a)
        y = dp_yield(P, Q, phi, c, sf)
        res = np.concatenate([e - e_tr + dl[:, None] * gg, y[:, None]], 1)
        Jm = np.zeros((e.shape[0], 4, 4), dtype=np.result_type(e, hge))
        Jm[:, :3, :3] = eye3 + dl[:, None, None] * hge
        Jm[:, :3, 3] = gg
        Jm[:, 3, :3] = gfe
        xd = np.linalg.solve(Jm, res[:, :, None])[:, :, 0]
        e = e - xd[:, :3]
        dl = dl - xd[:, 3]
        tau, P, S, Q = inv(e)
    K = lam_v + 2.0 * mu_v / 3.0
    e_apex = np.broadcast_to(p_tip / (3.0 * K), e_tr.shape)
    e = np.where(apex[:, None], e_apex, e)
    return np.where(elastic[:, None], e_tr, e)


# ---------------------------------------------------------------- NorSand
def _ns_eta(M, N, P, pi):
    if abs(N) < 1e-10:
        return M * (1.0 + np.log(pi / P))
    return (M / N) * (1.0 - (1.0 - N) * (P / pi) ** (N / (1.0 - N)))


def _ns_dEtadP(M, N, P, pi):
    if abs(N) < 1e-10:
        return M * (-1.0) / P
    return M * (-1.0 * (P / pi) ** ((2.0 * N - 1.0) / (1.0 - N)) / pi)


def _ns_dEtadPi(M, N, P, pi):
    if abs(N) < 1e-10:
        return M / pi
    return M * (-1.0 * (P / pi) ** ((2.0 * N - 1.0) / (1.0 - N)) * (-P) / pi ** 2)


def ns_eps_s(e):
    return np.sqrt(2.0 / 9.0 * ((e[:, 0] - e[:, 1]) ** 2 + (e[:, 1] - e[:, 2]) ** 2 + (e[:, 0] - e[:, 2]) ** 2))


def return_map_norsand(e_tr, eps_v_total, pi_old, pi_new_in, prm, tol=1e-10, n_local=15):
    """NorSand (Borja & Andrade 2006) return map, fixed n_local iterations.

    Follows return_mapping_NorSand, triaxial_NorSand.py:243-400.  prm holds
    kappa, tilde_lambda, M, N, beta, vc0, p0, v0, h, mu (G0) and eps_v0 (the
    reference's initial_volumetric_strain).  Returns (e_real, pi_new): pi_new
    is written only for plastic points; elsewhere pi_new_in is passed through,
    exactly as the reference leaves new_pi_array untouched (:398).
    """
    kap, tl, M, N = prm["kappa"], prm["tilde_lambda"], prm["M"], prm["N"]
    beta, vc0, p0, v0, h = prm["beta"], prm["vc0"], prm["p0"], prm["v0"], prm["h"]
    mu, ev0 = prm["mu"], prm["eps_v0"]
    ab = -3.5 / beta
    eps_v = e_tr.sum(1)
    eps_s = ns_eps_s(e_tr)
    big = np.real(eps_s) > tol
    with np.errstate(divide="ignore", invalid="ignore"):
        nd = np.sqrt(2.0 / 3.0) * (e_tr - eps_v[:, None] / 3.0) / eps_s[:, None]
    nd = np.where(big[:, None], nd, 0.0)
    P = p0 * np.exp(-(eps_v - ev0) / kap)
    Q = 3.0 * mu * eps_s
    new_v = np.exp(eps_v_total) * v0
    tension = np.real(eps_v) > tol
    y0 = Q + _ns_eta(M, N, P, pi_old) * P
    plastic = (~tension) & (np.real(y0) >= tol)

    e = e_tr.copy()
    pi = np.array(pi_old, dtype=np.result_type(pi_old, e_tr), copy=True)
    dl = np.zeros_like(eps_v)
    with np.errstate(all="ignore"):
        for _ in range(n_local):
            ev = e.sum(1)
            es = ns_eps_s(e)
            dEdP = _ns_dEtadP(M, N, P, pi)
            dEdPi = _ns_dEtadPi(M, N, P, pi)
            eta = _ns_eta(M, N, P, pi)
            dFdP = (eta - M) / (1.0 - N)
            dFdQ = 1.0
            psi_i = new_v - vc0 + tl * np.log(-pi)
            if abs(N) < tol:
                pistar = P * np.exp(ab * psi_i / M)
            else:
                pistar = P * (1.0 - ab * psi_i * N / M) ** ((N - 1.0) / N)
            y = Q + eta * P
            hard = pi - pi_old + h * (pi - pistar) * dl
            res = np.stack([ev - eps_v + dl * beta * dFdP, es - eps_s + dl * dFdQ, y, hard], 1)
            omn = -(ev - ev0) / kap
            dPde = p0 * np.exp(omn) / (-kap)
            d2F_dPdepsv = 1.0 / (1.0 - N) * dEdP * dPde
            d2F_dPdPi = 1.0 / (1.0 - N) * dEdPi
            dFdepsv = (dEdP * P + eta) * dPde
            dFdepss = 3.0 * mu
            dFdPi = P * dEdPi
            if abs(N) < 1e-10:
                dPs_dP = np.exp(ab * psi_i / M)
            else:
                dPs_dP = (1.0 - ab * psi_i * N / M) ** ((N - 1.0) / N)
            dPsii_dPi = tl / pi
            if abs(N) < 1e-10:
                dPs_dPi = P * np.exp(ab * psi_i / M) * ab / M * dPsii_dPi
            else:
                dPs_dPi = P * (N - 1.0) / N * (1.0 / (1.0 - ab * psi_i * N / M)) ** (1.0 / N) * (-ab * N / M) * dPsii_dPi
            dHdepsv = -h * dl * dPs_dP * dPde
            dHdPi = 1.0 + h * dl * (1.0 - dPs_dPi)
            n = e.shape[0]
            Jm = np.zeros((n, 4, 4), dtype=np.result_type(e, pi, dFdepsv))
            Jm[:, 0, 0] = 1.0 + dl * beta * d2F_dPdepsv
            Jm[:, 0, 2] = beta * dFdP
            Jm[:, 0, 3] = dl * beta * d2F_dPdPi
            Jm[:, 1, 1] = 1.0
            Jm[:, 1, 2] = dFdQ
            Jm[:, 2, 0] = dFdepsv
            Jm[:, 2, 1] = dFdepss
            Jm[:, 2, 3] = dFdPi
            Jm[:, 3, 0] = dHdepsv
            Jm[:, 3, 2] = h * (pi - pistar)
            Jm[:, 3, 3] = dHdPi
            # Elastic points would make Jm singular; solve them on identity.
            Jm = np.where(plastic[:, None, None], Jm, np.eye(4))
            xd = np.linalg.solve(Jm, res[:, :, None])[:, :, 0]
            nev = ev - xd[:, 0]
            nes = es - xd[:, 1]
            dl = dl - xd[:, 2]
            pi = pi - xd[:, 3]
            e = nev[:, None] / 3.0 + nes[:, None] * nd * np.sqrt(1.5)
            P = p0 * np.exp(-(e.sum(1) - ev0) / kap)
            Q = 3.0 * mu * ns_eps_s(e)
    e_out = np.where(plastic[:, None], e, e_tr)
    e_out = np.where(tension[:, None], 0.0, e_out)
    pi_out = np.where(plastic, pi, pi_new_in)
    return e_out, pi_out


def kirchhoff_norsand(e, prm):
    """Pressure-dependent hyperelasticity (triaxial_NorSand.py:452-460)."""
    tr = e.sum(1, keepdims=True)
    om = -(tr - prm["eps_v0"]) / prm["kappa"]
    return -prm["p0"] * prm["kappa"] * np.exp(om) / (-prm["kappa"]) + 2.0 / 3.0 * prm["mu"] * (3.0 * e - tr)
