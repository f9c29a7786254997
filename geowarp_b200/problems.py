"""Problem setups built on the drop-in solver classes.

Each builder returns a solver object configured the way the reference's
problem scripts configure theirs (dicts + Dirichlet flags), at the sizes of the
benchmark workloads:

  strip_footing_2d   plane-strain rigid strip footing on Drucker-Prager soil
                     (a 2D restatement of the 3D penalty indenter of
                     problems/3D_indentation/3d_indentation_coupled_cpGIMP.py)
  bar_compaction_2d  bar under self-weight (problems/bar_compaction/bar_compaction_cpGIMP.py)
"""
import numpy as np
import torch

from .solvers.quasi_static_solver_2d import quasi_static_solver_2d


def strip_footing_dicts(n_cells_x=256, n_cells_y=128, dx=0.05, PPD=2, E=2e7, nu=0.3, cohesion=1e4,
                        friction_angle=30.0, dilation_angle=0.0, footing_width=1.0, total_disp=0.2, n_steps=100,
                        penalty_factor=1000.0, rho=2000.0, gravity=9.81, n_iter=30, tol=1e-6, pad=2):
    """Soil block of n_cells_x x n_cells_y cells (PPD^2 particles per cell) in a
    grid padded by `pad` cells on every side; footing centred on the top.

    The footing starts at the height of the top particle layer and each load
    step lowers it by total_disp / n_steps.  Its penalty acts as an attractive
    spring (footing_penalty_stable): the reference's 3D indenter residual
    k (z_new - h) (mpm/mpm_utils.py:1243-1245) is a repulsive spring whose
    negative stiffness the Drucker-Prager soil cannot stabilise here, and the
    Drucker-Prager map continues past the cone tip (tension_cutoff=False).

    The soil has self-weight at full magnitude from the first load step
    (gravity_ramp=False) and starts from the matching geostatic stress
    (geostatic_stress below).  Without it (gravity=0) the unconfined column
    under a 1 m footing yields through ~3 m of depth at ~170 kPa and the
    Newton iteration meets a near-mechanism after ~12 mm of footing travel."""
    n_grid_x, n_grid_y = n_cells_x + 2 * pad, n_cells_y + 2 * pad
    start_x, start_y = pad * dx, pad * dx
    end_x, end_y = start_x + n_cells_x * dx, start_y + n_cells_y * dx
    grid = dict(n_grid_x=n_grid_x, n_grid_y=n_grid_y, max_x=n_grid_x * dx, dx=dx, start_x=start_x, end_x=end_x,
                start_y=start_y, end_y=end_y, domain_min_x=start_x, domain_max_x=end_x, domain_min_y=start_y,
                domain_max_y=end_y)
    parts = dict(n_particles=n_cells_x * n_cells_y * PPD * PPD, PPD=PPD, p_vol=(dx / PPD) ** 2, p_rho=rho)
    it = dict(n_iter=n_iter, tol=tol, solver_name="warp")
    mat = dict(youngs_modulus=E, poisson_ratio=nu, material_name="Drucker-Prager", friction_angle=friction_angle,
               dilation_angle=dilation_angle, cohesion=cohesion, shape_factor=0.0, tension_cutoff=False)
    xc = 0.5 * (start_x + end_x)
    load = dict(gravity_mag=gravity, traction_value_x=0.0, traction_value_y=0.0, point_load_value_x=0.0,
                point_load_value_y=0.0, footing_region_min_x=xc - footing_width / 2,
                footing_region_max_x=xc + footing_width / 2, footing_initial_height=end_y - dx / (2 * PPD),
                footing_incr_disp=-total_disp / n_steps, penalty_factor=penalty_factor, footing_penalty_stable=True,
                gravity_ramp=False)
    return grid, parts, it, mat, load


def strip_footing_boundary(grid):
    """Rollers on the side walls (x fixed), fixed base (x, y fixed): field-major flags."""
    nx, ny, dx = grid["n_grid_x"], grid["n_grid_y"], grid["dx"]
    nn = (nx + 1) * (ny + 1)
    ix = np.tile(np.arange(nx + 1), ny + 1)
    iy = np.repeat(np.arange(ny + 1), nx + 1)
    dof = ix + iy * (nx + 1)
    i0 = int(round(grid["start_x"] / dx))
    i1 = int(round(grid["end_x"] / dx))
    j0 = int(round(grid["start_y"] / dx))
    b = np.zeros(2 * nn, dtype=bool)
    side = (ix <= i0) | (ix >= i1)
    base = iy <= j0
    b[dof[side | base]] = True
    b[dof[base] + nn] = True
    return b


def geostatic_left_cauchy_green(y, surface_y, rho, gravity, E, nu, K0):
    """Elastic left Cauchy-Green tensors b (N x 3 x 3) of a geostatic state:
    sigma_yy = -rho g (surface_y - y), sigma_xx = sigma_zz = K0 sigma_yy, no
    shear.  Inverts the Hencky law tau = lam tr(eps) I + 2 mu eps with
    eps = log(b) / 2 and tau = sigma (J = 1 at the start)."""
    y = torch.as_tensor(y, dtype=torch.float64)
    E = torch.as_tensor(E, dtype=torch.float64, device=y.device)
    E = E.reshape(-1, 1) if E.dim() else E  # per-particle moduli broadcast over the 3 axes
    lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    mu = E / (2.0 * (1.0 + nu))
    syy = -rho * gravity * (surface_y - y)
    tau = torch.stack([K0 * syy, syy, K0 * syy], dim=-1)
    tr_eps = tau.sum(-1, keepdim=True) / (3.0 * lam + 2.0 * mu)
    eps = (tau - lam * tr_eps) / (2.0 * mu)
    return torch.diag_embed(torch.exp(2.0 * eps))


def geostatic_stress(solver, surface_y, rho, gravity, K0):
    """Start a 2D solid solver from the geostatic state of a soil layer whose
    top is at surface_y: sets the elastic left Cauchy-Green tensors (old and
    new) and the Cauchy stress of every particle."""
    e = solver.engine
    E = e.E if e.E is not None else solver.youngs_modulus
    b = geostatic_left_cauchy_green(e.x[:, 1], surface_y, rho, gravity, E, solver.poisson_ratio, K0)
    e.b_old.copy_(b)
    e.b_new.copy_(b)
    syy = -rho * gravity * (surface_y - e.x[:, 1])
    e.sigma.zero_()
    e.sigma[:, 0, 0] = K0 * syy
    e.sigma[:, 1, 1] = syy
    e.sigma[:, 2, 2] = K0 * syy


def strip_footing_2d(precision="fp64", device=None, K0=None, **kw):
    grid, parts, it, mat, load = strip_footing_dicts(**kw)
    s = quasi_static_solver_2d(grid, parts, it, mat, load, precision=precision, device=device)
    s.engine.line_search_growth = 2.0  # safeguard for the growing plastic zone
    s.dofStruct.boundary_flag_array[:] = torch.as_tensor(strip_footing_boundary(grid),
                                                        device=s.x_particles.device)
    if load["gravity_mag"] > 0.0:
        if K0 is None:  # Jaky's at-rest coefficient
            K0 = 1.0 - np.sin(np.radians(mat["friction_angle"]))
        geostatic_stress(s, grid["end_y"], parts["p_rho"], load["gravity_mag"], K0)
    return s
