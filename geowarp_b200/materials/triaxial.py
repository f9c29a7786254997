"""Strain-driven triaxial material tests on the GPU.

The drivers of problems/material_tests/triaxial_DruckerPrager.py:497-611 and
problems/material_tests/triaxial_NorSand.py:497-628: initial strain from the
isotropic elastic stiffness and the target stresses, an axial strain
increment per step, and a Newton iteration on the two radial strains so the
radial stresses meet their targets.  The return map and its algorithmic
tangent (the Jacobian the reference obtains from its 6x6 tape) are evaluated
by the engine's CUDA return-map kernel.
"""
import numpy as np
import torch

from .plasticity import return_mapping


def _lame(E, nu):
    return E * nu / ((1 + nu) * (1 - 2 * nu)), E / (2 * (1 + nu))


def _initial_strain(target, lam, mu):
    C = lam * np.ones((3, 3)) + 2 * mu * np.eye(3)
    return np.linalg.solve(C, np.asarray(target, dtype=np.float64))


def _run(md, trial, total, target, n_steps, rate, device, ns_state=None, tol=1e-10, n_iter=10):
    P, Q, vol = [], [], []
    ev0 = total.sum()
    for _ in range(n_steps):
        trial = trial.copy()
        total = total.copy()
        trial[2] -= rate
        total[2] -= rate
        for _it in range(n_iter):
            kw = {}
            if ns_state is not None:
                kw = dict(eps_v_total=torch.tensor([total.sum()], dtype=torch.float64, device=device),
                          pi_old=torch.tensor([ns_state[0]], dtype=torch.float64, device=device),
                          pi_new=torch.tensor([ns_state[1]], dtype=torch.float64, device=device))
            e, tau, dt, pn = return_mapping(md, torch.tensor(trial[None, :], dtype=torch.float64, device=device), tangent=True, **kw)
            s = tau[0].cpu().numpy()
            rhs = np.array([target[0] - s[0], target[1] - s[1]])
            J = -dt[0].cpu().numpy()[:2, :2]
            inc = np.linalg.solve(J, rhs)
            trial[:2] -= inc
            total[:2] -= inc
            if np.linalg.norm(rhs) < tol:
                break
        kw = {}
        if ns_state is not None:
            kw = dict(eps_v_total=torch.tensor([total.sum()], dtype=torch.float64, device=device),
                      pi_old=torch.tensor([ns_state[0]], dtype=torch.float64, device=device),
                      pi_new=torch.tensor([ns_state[1]], dtype=torch.float64, device=device))
        e, tau, _, pn = return_mapping(md, torch.tensor(trial[None, :], dtype=torch.float64, device=device), **kw)
        s = tau[0].cpu().numpy()
        if ns_state is not None:
            ns_state = (float(pn[0]), float(pn[0]))
        P.append(-(s[0] + s[1] + s[2]) / 3.0)
        Q.append(-s[2] - (-s[0]))
        vol.append(-total.sum() * 100.0 + ev0 * 100.0)
        trial = e[0].cpu().numpy().copy()
    return np.array(P), np.array(Q), np.array(vol)


def triaxial_DruckerPrager(E=25000.0, nu=0.3, friction_angle=35.0, dilation_angle=5.0, cohesion=0.0,
                           shape_factor=0.0, final_axial_strain=0.1, n_steps=100, confining=-150.0, axial=-150.0,
                           device="cuda"):
    """(P, Q) per step, as printed by triaxial_DruckerPrager.py:606-611."""
    lam, mu = _lame(E, nu)
    target = np.array([confining, confining, axial])
    trial = _initial_strain(target, lam, mu)
    md = dict(material_name="Drucker-Prager", youngs_modulus=E, poisson_ratio=nu, friction_angle=friction_angle,
              dilation_angle=dilation_angle, cohesion=cohesion, shape_factor=shape_factor)
    P, Q, _ = _run(md, trial, trial.copy(), target, n_steps, final_axial_strain / n_steps, device)
    return P, Q


def triaxial_NorSand(G0=4.5e4, kappa=0.0015, tilde_lambda=0.02, M=1.27, N=0.4, beta=1.0, vc0=1.8911, pc=-715.0,
                     p0=-390.0, v0=1.75, h=70.0, K0_consolidation=0.45, final_axial_strain=0.1, n_steps=500,
                     device="cuda"):
    """(axial strain %, Q, volumetric strain %) per step (triaxial_NorSand.py:615-628)."""
    K0 = p0 / (-kappa)
    lam, mu = K0 - 2.0 / 3.0 * G0, G0
    E = mu * (3 * lam + 2 * mu) / (lam + mu)
    nu = lam / (2 * (lam + mu))
    slope = (1.0 - K0_consolidation) / (1.0 / 3.0 * (1.0 + 2.0 * K0_consolidation))
    txx = (3.0 - slope) / 3.0 * p0
    target = np.array([txx, txx, (3.0 + 2 * slope) / 3.0 * p0])
    trial = _initial_strain(target, lam, mu)
    pi0 = pc * (1.0 - N) ** ((1.0 - N) / N)
    md = dict(material_name="NorSand", youngs_modulus=E, poisson_ratio=nu, kappa=kappa, tilde_lambda=tilde_lambda,
              M=M, N=N, beta=beta, vc0=vc0, p0=p0, v0=v0, h=h, shear_modulus=G0,
              initial_volumetric_strain=float(trial.sum()))
    rate = final_axial_strain / n_steps
    _, Q, vol = _run(md, trial, trial.copy(), target, n_steps, rate, device, ns_state=(pi0, pi0))
    ax = (np.arange(n_steps) + 1) * rate * 100.0
    return ax, Q, vol
