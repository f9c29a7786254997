"""GPU parity: single-point return maps and their algorithmic tangents against the oracle."""
import numpy as np
import pytest
import torch

from oracle import materials as MT

pytestmark = pytest.mark.gpu

NS = dict(kappa=0.0015, tilde_lambda=0.02, M=1.27, N=0.4, beta=1.0, vc0=1.8911, p0=-390.0, v0=1.75, h=70.0,
          shear_modulus=4.5e4, initial_volumetric_strain=0.0)


def lame(E, nu):
    return E * nu / ((1 + nu) * (1 - 2 * nu)), E / (2 * (1 + nu))


def cs_tangent(fn, e, h=1e-30):
    out = []
    for b in range(3):
        ec = e.astype(np.complex128)
        ec[:, b] += 1j * h
        out.append(np.imag(fn(ec)) / h)
    return np.stack(out, 2)  # [n, A, B]


def test_dp_return_map(cuda):
    from geowarp_b200.materials.plasticity import return_mapping
    rng = np.random.default_rng(0)
    E, nu, phi, psi, c = 2.5e4, 0.3, 35.0, 5.0, 2.0
    lam, mu = lame(E, nu)
    e = rng.normal(scale=0.01, size=(512, 3)) - 0.004
    md = dict(material_name="Drucker-Prager", youngs_modulus=E, poisson_ratio=nu, friction_angle=phi,
              dilation_angle=psi, cohesion=c)
    eg, tg, dg, _ = return_mapping(md, torch.as_tensor(e, device=cuda), tangent=True)
    eo = MT.return_map_dp(e, lam, mu, phi, psi, c, 0.0)
    to = MT.kirchhoff_hencky(eo, lam, mu)
    do = cs_tangent(lambda z: MT.kirchhoff_hencky(MT.return_map_dp(z, lam, mu, phi, psi, c, 0.0), lam, mu), e)
    assert np.abs(eg.cpu().numpy() - eo).max() < 1e-12
    assert np.abs(tg.cpu().numpy() - to).max() < 1e-9 * np.abs(to).max()
    assert np.abs(dg.cpu().numpy() - do).max() < 1e-8 * np.abs(do).max()


def test_j2_return_map(cuda):
    from geowarp_b200.materials.plasticity import return_mapping
    rng = np.random.default_rng(1)
    E, nu, kappa = 10.0, 0.0, 5.0
    lam, mu = lame(E, nu)
    e = rng.normal(scale=0.5, size=(256, 3))
    md = dict(material_name="J2", youngs_modulus=E, poisson_ratio=nu, kappa=kappa)
    eg, tg, dg, _ = return_mapping(md, torch.as_tensor(e, device=cuda), tangent=True)
    eo = MT.return_map_j2(e, lam, mu, kappa)
    do = cs_tangent(lambda z: MT.kirchhoff_hencky(MT.return_map_j2(z, lam, mu, kappa), lam, mu), e)
    assert np.abs(eg.cpu().numpy() - eo).max() < 1e-13
    assert np.abs(dg.cpu().numpy() - do).max() < 1e-9 * np.abs(do).max()


def test_norsand_return_map(cuda):
    """Physical states: the K0-consolidated loose Brasted sand of
    triaxial_NorSand.py:23-52 with small compressive / deviatoric increments."""
    from geowarp_b200.materials.plasticity import return_mapping
    from oracle.triaxial import NORSAND_LOOSE as P0, initial_strain
    rng = np.random.default_rng(2)
    n = 256
    K0 = P0["p0"] / (-P0["kappa"])
    lam, mu = K0 - 2.0 / 3.0 * P0["G0"], P0["G0"]
    slope = (1.0 - P0["K0_consolidation"]) / (1.0 / 3.0 * (1.0 + 2.0 * P0["K0_consolidation"]))
    txx = (3.0 - slope) / 3.0 * P0["p0"]
    e0 = initial_strain([txx, txx, (3.0 + 2 * slope) / 3.0 * P0["p0"]], lam, mu)
    ev0 = e0.sum()
    e = e0[None, :] + np.stack([rng.uniform(0, 4e-4, n), rng.uniform(0, 4e-4, n), -rng.uniform(0, 3e-3, n)], 1)
    evt = e.sum(1)
    pi0 = P0["pc"] * (1 - P0["N"]) ** ((1 - P0["N"]) / P0["N"])
    pi_old = np.full(n, pi0)
    md = dict(material_name="NorSand", kappa=P0["kappa"], tilde_lambda=P0["tilde_lambda"], M=P0["M"], N=P0["N"],
              beta=P0["beta"], vc0=P0["vc0"], p0=P0["p0"], v0=P0["v0"], h=P0["h"], shear_modulus=P0["G0"],
              initial_volumetric_strain=ev0)
    eg, tg, _, png = return_mapping(md, torch.as_tensor(e, device=cuda),
                                    eps_v_total=torch.as_tensor(evt, device=cuda),
                                    pi_old=torch.as_tensor(pi_old, device=cuda),
                                    pi_new=torch.as_tensor(pi_old, device=cuda))
    prm = dict(kappa=P0["kappa"], tilde_lambda=P0["tilde_lambda"], M=P0["M"], N=P0["N"], beta=P0["beta"],
               vc0=P0["vc0"], p0=P0["p0"], v0=P0["v0"], h=P0["h"], mu=P0["G0"], eps_v0=ev0)
    eo, po = MT.return_map_norsand(e, evt, pi_old, pi_old.copy(), prm)
    to = MT.kirchhoff_norsand(eo, prm)
    assert (po != pi0).sum() > n // 4  # a good share of the points is plastic
    assert np.abs(eg.cpu().numpy() - eo).max() < 1e-12
    assert np.abs(tg.cpu().numpy() - to).max() < 1e-9 * np.abs(to).max()
    assert np.abs(png.cpu().numpy() - po).max() < 1e-10 * np.abs(po).max()


def test_triaxial_paths_match_golden(cuda):
    """Full strain-driven triaxial tests on the GPU against the oracle's curves."""
    import os
    from geowarp_b200.materials.triaxial import triaxial_DruckerPrager, triaxial_NorSand
    gdir = os.path.join(os.path.dirname(__file__), "golden")
    g = np.load(os.path.join(gdir, "triaxial_dp.npz"))
    P, Q = triaxial_DruckerPrager(device=cuda)
    assert np.abs(P - g["P"]).max() < 1e-8 * np.abs(g["P"]).max()
    assert np.abs(Q - g["Q"]).max() < 1e-8 * np.abs(g["Q"]).max()
    g = np.load(os.path.join(gdir, "triaxial_norsand.npz"))
    ax, Qn, vol = triaxial_NorSand(n_steps=100, device=cuda)
    assert np.abs(Qn - g["Q"]).max() < 1e-7 * np.abs(g["Q"]).max()
    assert np.abs(vol - g["vol"]).max() < 1e-7 * max(np.abs(g["vol"]).max(), 1e-12)
