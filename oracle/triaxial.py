"""Strain-driven triaxial tests of the return maps (oracle).

Restates the drivers problems/material_tests/triaxial_DruckerPrager.py:497-611
and problems/material_tests/triaxial_NorSand.py:497-628: an initial strain
from the isotropic elastic stiffness and the target stresses, then per step an
axial strain increment and a global Newton on the two radial strains so that
the radial stresses match their targets (tol 1e-10, at most 10 iterations),
after which the elastic strain becomes the next trial strain.  The reference's
6x6 tape Jacobian has nonzero rows only for the two radial residuals; a
central-difference 2x2 Jacobian reaches the same converged states.
"""
import numpy as np

from . import materials as MT


def _lame(E, nu):
    return E * nu / ((1 + nu) * (1 - 2 * nu)), E / (2 * (1 + nu))


def initial_strain(target, lam, mu):
    """Normal strains of C^-1 sigma_target for isotropic C (Voigt, normal block)."""
    C = lam * np.ones((3, 3)) + 2 * mu * np.eye(3)
    return np.linalg.solve(C, np.asarray(target, dtype=np.float64))


def _newton(stress_fn, trial, total, target_xy, tol=1e-10, n_iter=10):
    for _ in range(n_iter):
        s, extra = stress_fn(trial, total)
        rhs = np.array([target_xy[0] - s[0], target_xy[1] - s[1]])
        J = np.zeros((2, 2))
        h = 1e-9
        for c in range(2):
            tp, tm = trial.copy(), trial.copy()
            tp[c] += h
            tm[c] -= h
            sp_, _ = stress_fn(tp, total)
            sm_, _ = stress_fn(tm, total)
            J[:, c] = -(sp_[:2] - sm_[:2]) / (2 * h)  # d rhs / d trial
        inc = np.linalg.solve(J, rhs)
        trial = trial.copy()
        total = total.copy()
        trial[:2] -= inc
        total[:2] -= inc
        if np.linalg.norm(rhs) < tol:
            break
    return trial, total, s, extra


def triaxial_dp(E=25000.0, nu=0.3, phi=35.0, psi=5.0, c=0.0, sf=0.0, final_axial_strain=0.1, n_steps=100,
                confining=-150.0, axial=-150.0, tension_cutoff=True):
    """Returns (P[n_steps], Q[n_steps], e_trial_history[n_steps, 3]) as the reference prints them."""
    lam, mu = _lame(E, nu)
    rate = final_axial_strain / n_steps
    target = np.array([confining, confining, axial])
    trial = initial_strain(target, lam, mu)
    total = trial.copy()

    def stress(tr, to):
        e = MT.return_map_dp(tr[None, :], lam, mu, phi, psi, c, sf, tension_cutoff=tension_cutoff)[0]
        return MT.kirchhoff_hencky(e[None, :], lam, mu)[0], e

    P, Q, hist = [], [], []
    for _ in range(n_steps):
        trial = trial.copy()
        total = total.copy()
        trial[2] -= rate
        total[2] -= rate
        trial, total, s, e = _newton(stress, trial, total, target[:2])
        hist.append(trial.copy())
        s, e = stress(trial, total)
        P.append(-(s[0] + s[1] + s[2]) / 3.0)
        Q.append(-s[2] - (-s[0]))
        trial = e.copy()  # set_new_trial_strain_array_to_elastic_strain
    return np.array(P), np.array(Q), np.array(hist)


NORSAND_LOOSE = dict(G0=4.5e4, kappa=0.0015, tilde_lambda=0.02, M=1.27, N=0.4, beta=1.0, vc0=1.8911,
                     pc=-715.0, p0=-390.0, v0=1.75, h=70.0, K0_consolidation=0.45)


def triaxial_norsand(prm=NORSAND_LOOSE, final_axial_strain=0.1, n_steps=500):
    """NorSand triaxial (loose Brasted sand of triaxial_NorSand.py:13-43).
    Returns (axial_strain_percent, Q, volumetric_strain_percent)."""
    N = prm["N"]
    pi0 = prm["pc"] * (1.0 - N) ** ((1.0 - N) / N)
    K0 = prm["p0"] / (-prm["kappa"])
    lam = K0 - 2.0 / 3.0 * prm["G0"]
    mu = prm["G0"]
    rate = final_axial_strain / n_steps
    k0c = prm["K0_consolidation"]
    slope = (1.0 - k0c) / (1.0 / 3.0 * (1.0 + 2.0 * k0c))
    txx = (3.0 - slope) / 3.0 * prm["p0"]
    tzz = (3.0 + 2 * slope) / 3.0 * prm["p0"]
    target = np.array([txx, txx, tzz])
    trial = initial_strain(target, lam, mu)
    total = trial.copy()
    ev0 = total.sum()
    mprm = dict(kappa=prm["kappa"], tilde_lambda=prm["tilde_lambda"], M=prm["M"], N=N, beta=prm["beta"],
                vc0=prm["vc0"], p0=prm["p0"], v0=prm["v0"], h=prm["h"], mu=mu, eps_v0=ev0)
    state = dict(pi_old=np.array([pi0]), pi_new=np.array([pi0]))

    def stress(tr, to):
        e, pn = MT.return_map_norsand(tr[None, :], np.array([to.sum()]), state["pi_old"], state["pi_new"], mprm)
        return MT.kirchhoff_norsand(e, mprm)[0], (e[0], pn)

    ax, Qs, vol = [], [], []
    for step in range(n_steps):
        trial = trial.copy()
        total = total.copy()
        trial[2] -= rate
        total[2] -= rate
        trial, total, s, (e, pn) = _newton(stress, trial, total, target[:2])
        s, (e, pn) = stress(trial, total)
        state["pi_new"] = pn  # new_pi_array keeps the last plastic value
        state["pi_old"] = state["pi_new"].copy()
        trial = e.copy()
        ax.append((step + 1) * rate * 100.0)
        Qs.append(-s[2] - (-s[0]))
        vol.append(-1.0 * total.sum() * 100.0 - (-ev0 * 100.0))
    return np.array(ax), np.array(Qs), np.array(vol)
