"""Return maps in principal log-strain space, evaluated on the GPU.

Batched entry points over n material points (torch tensors, float64, CUDA)
for the three plastic models of the engine: J2 (materials/plasticity.py:8-37),
Drucker-Prager (problems/material_tests/triaxial_DruckerPrager.py:119-412) and
NorSand (problems/material_tests/triaxial_NorSand.py:155-400).  Each returns
the corrected principal strains, the principal Kirchhoff stresses and, on
request, the algorithmic tangent d tau_A / d e_trial_B (exact derivative of
the fixed-count local iteration).  The MPM kernels call the same device code.
"""
import ctypes as C

import torch

from .. import _lib as L
from ..engine import material_struct


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)


def return_mapping(material_dict, e_trial, eps_v_total=None, pi_old=None, pi_new=None, tangent=False):
    """Evaluate the model of material_dict at principal trial strains e_trial [n, 3].

    Returns (e_real [n,3], tau [n,3], dtau_de [n,3,3] or None, pi_new [n] or None).
    """
    e_trial = e_trial.to(torch.float64).contiguous()
    n = e_trial.shape[0]
    dev = e_trial.device
    f64 = lambda t: None if t is None else torch.as_tensor(t, device=dev).to(torch.float64).reshape(-1).contiguous()
    eps_v_total, pi_old, pi_new = f64(eps_v_total), f64(pi_old), f64(pi_new)
    m = material_struct(material_dict)
    e_out = torch.empty_like(e_trial)
    tau = torch.empty_like(e_trial)
    dtau = torch.empty((n, 3, 3), dtype=torch.float64, device=dev) if tangent else None
    pn = None
    if pi_new is not None:
        pn = pi_new.clone().contiguous()
    L.call("gw_return_map", C.byref(m), n, _ptr(e_trial), _ptr(eps_v_total), _ptr(pi_old), _ptr(pn), _ptr(e_out),
           _ptr(tau), _ptr(dtau), C.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    return e_out, tau, dtau, pn


def return_mapping_J2(e_trial, lame_lambda, lame_mu, kappa, tangent=False):
    E = lame_mu * (3 * lame_lambda + 2 * lame_mu) / (lame_lambda + lame_mu)
    nu = lame_lambda / (2 * (lame_lambda + lame_mu))
    md = dict(material_name="J2", youngs_modulus=E, poisson_ratio=nu, kappa=kappa)
    return return_mapping(md, e_trial, tangent=tangent)[:3:2] if tangent else return_mapping(md, e_trial)[0]


def return_mapping_DruckerPrager(e_trial, youngs_modulus, poisson_ratio, friction_angle, dilation_angle, cohesion,
                                 shape_factor=0.0, tangent=False):
    md = dict(material_name="Drucker-Prager", youngs_modulus=youngs_modulus, poisson_ratio=poisson_ratio,
              friction_angle=friction_angle, dilation_angle=dilation_angle, cohesion=cohesion,
              shape_factor=shape_factor)
    e, tau, dt, _ = return_mapping(md, e_trial, tangent=tangent)
    return (e, tau, dt) if tangent else e


def return_mapping_NorSand(e_trial, eps_v_total, pi_old, pi_new, params, tangent=False):
    """params: kappa, tilde_lambda, M, N, beta, vc0, p0, v0, h, shear_modulus,
    initial_volumetric_strain (names of triaxial_NorSand.py:13-43)."""
    md = dict(material_name="NorSand", **params)
    return return_mapping(md, e_trial, eps_v_total=eps_v_total.contiguous(), pi_old=pi_old.contiguous(),
                          pi_new=pi_new, tangent=tangent)
