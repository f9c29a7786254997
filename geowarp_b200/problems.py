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


# ---------------------------------------------------------------- bar compaction (self-weight)
def bar_compaction_2d(precision="fp64", device=None, width_cells=4, height_cells=40, dx=0.25, PPD=2, E=1e6, nu=0.3,
                      rho=80.0, gravity=9.81, material="Neo-Hookean", n_iter=20, tol=1e-6, precond="mg"):
    """A bar width_cells x height_cells cells under self-weight ramped over the
    load steps (problems/bar_compaction/bar_compaction_cpGIMP.py): rollers on
    both side walls, fixed base, two empty cells around it."""
    pad = 2
    n_grid_x, n_grid_y = width_cells + 2 * pad, height_cells + 2 * pad
    sx, sy = pad * dx, pad * dx
    ex, ey = sx + width_cells * dx, sy + height_cells * dx
    grid = dict(n_grid_x=n_grid_x, n_grid_y=n_grid_y, max_x=n_grid_x * dx, dx=dx, start_x=sx, end_x=ex,
                start_y=sy, end_y=ey, domain_min_x=sx, domain_max_x=ex, domain_min_y=sy, domain_max_y=ey)
    parts = dict(n_particles=width_cells * height_cells * PPD * PPD, PPD=PPD, p_vol=(dx / PPD) ** 2, p_rho=rho)
    it = dict(n_iter=n_iter, tol=tol, solver_name="warp")
    mat = dict(youngs_modulus=E, poisson_ratio=nu, material_name=material)
    load = dict(gravity_mag=gravity, traction_value_x=0.0, traction_value_y=0.0, point_load_value_x=0.0,
                point_load_value_y=0.0)
    s = quasi_static_solver_2d(grid, parts, it, mat, load, precision=precision, device=device, precond=precond)
    nx1 = n_grid_x + 1
    nn = nx1 * (n_grid_y + 1)
    ix = np.tile(np.arange(nx1), n_grid_y + 1)
    iy = np.repeat(np.arange(n_grid_y + 1), nx1)
    b = np.zeros(2 * nn, dtype=bool)
    b[((ix <= pad) | (ix >= pad + width_cells)).nonzero()[0]] = True
    b[(iy <= pad).nonzero()[0]] = True
    b[(iy <= pad).nonzero()[0] + nn] = True
    s.dofStruct.boundary_flag_array[:] = torch.as_tensor(b, device=s.x_particles.device)
    return s


# ---------------------------------------------------------------- 1D consolidation (u-p)
def terzaghi_pressure(z_from_drained, t, H, cv, q, terms=200):
    """Terzaghi's excess pore pressure in a layer of height H drained on one
    face and undrained on the other, under a sudden surface load q:
    p = q sum_m (2/M) sin(M z/H) exp(-M^2 T),  M = pi (2m+1)/2,  T = cv t / H^2."""
    z = np.asarray(z_from_drained, dtype=np.float64)
    T = cv * t / H ** 2
    p = np.zeros_like(z)
    for m in range(terms):
        M = np.pi * (2 * m + 1) / 2
        p += 2.0 / M * np.sin(M * z / H) * np.exp(-M * M * T)
    return q * p


def consolidation_dts(n_steps, dt_first, t_end):
    """n_steps geometrically growing time increments dt_first r^k summing to t_end."""
    if dt_first * n_steps >= t_end:
        raise ValueError("dt_first * n_steps must stay below t_end")
    lo, hi = 1.0, 2.0
    while dt_first * (hi ** n_steps - 1) / (hi - 1) < t_end:
        hi *= 2.0
    for _ in range(200):
        r = 0.5 * (lo + hi)
        if dt_first * (r ** n_steps - 1) / (r - 1) < t_end:
            lo = r
        else:
            hi = r
    dts = dt_first * (0.5 * (lo + hi)) ** np.arange(n_steps)
    return dts * (t_end / dts.sum())


def consolidation_column_dicts(n_cells=200, dx=0.05, PPD=2, E=1e7, nu=0.3, permeability=1e-10, viscosity=1e-3,
                               porosity=0.4, surface_load=1e4, n_steps=200, first_fourier=4.0, T_end=2.0, n_iter=15,
                               tol=1e-8, material="Linear elasticity"):
    """Constructor dictionaries of the consolidation column (the layout of
    problems/consolidation/terzaghi_cpGIMP.py:10-73) plus its time
    increments: returns (grid, particles, iteration, material, porous, load,
    dts, cv, H)."""
    n_grid_x, n_grid_y = 6, n_cells + 2
    max_y = n_grid_y * dx
    sx, ex, sy, ey = dx, 2 * dx, 0.0, n_cells * dx
    grid = dict(n_grid_x=n_grid_x, n_grid_y=n_grid_y, max_x=n_grid_x * dx, dx=dx, max_y=max_y, dy=max_y / n_grid_y,
                start_x=sx, end_x=ex, start_y=sy, end_y=ey, domain_min_x=sx, domain_max_x=ex, domain_min_y=sy,
                domain_max_y=max_y)
    parts = dict(n_particles=n_cells * PPD * PPD, PPD=PPD, p_vol=(dx / PPD) ** 2, p_rho=1.0)
    H = n_cells * dx
    mobility = permeability / viscosity
    M = E * (1 - nu) / ((1 + nu) * (1 - 2 * nu))   # constrained modulus
    cv = mobility * M
    dts = consolidation_dts(n_steps, first_fourier * dx * dx / cv, T_end * H * H / cv)
    it = dict(n_iter=n_iter, tol=tol, solver_name="scipy", dt=float(dts[0]))
    mat = dict(youngs_modulus=E, poisson_ratio=nu, material_name=material)
    porous = dict(phi_initial=porosity, mobility_constant=mobility)
    load = dict(gravity_mag=0.0, traction_value_x=0.0, traction_value_y=-surface_load, point_load_value_x=0.0,
                point_load_value_y=0.0)
    return grid, parts, it, mat, porous, load, dts, cv, H


def consolidation_boundary_dofs(tid, boundary_flag_array, n_grid_x, n_nodes):
    """set_boundary_dofs of terzaghi_cpGIMP.py:104-119 on index tensors:
    x fixed on the side-wall node columns, y fixed on the base row."""
    ix, iy = tid
    dof_x = ix + iy * (n_grid_x + 1)
    boundary_flag_array[dof_x[(ix <= 1) | (ix >= 2)]] = True
    boundary_flag_array[dof_x[iy <= 0] + n_nodes] = True


def consolidation_column_2d(precision="fp64", device=None, precond="mg", krylov_rtol=None, **kw):
    """One-dimensional consolidation in a column of 1 x n_cells cells
    (problems/consolidation/terzaghi_cpGIMP.py): linear elastic skeleton,
    mobility k / mu, drained top with the surface load applied as a traction,
    undrained fixed base, rollers on the sides.  The n_steps time increments
    grow geometrically from a mesh Fourier number cv dt / dx^2 of
    first_fourier up to a Terzaghi time factor T_end = cv t / H^2 in total
    (keywords of consolidation_column_dicts); returns (solver, dts, cv, H).

    The Newton system is a saddle point (u-p) solved by flexible GMRES with
    the multigrid V-cycle (Schur-diagonal pressure smoother); node-block
    Jacobi Krylov stalls on it.  Increments far below one mesh Fourier number
    make it near-undrained and ill-conditioned for any smoother.  The FP64
    Krylov tolerance defaults to 1e-10, the reference's BiCGSTAB tolerance:
    1e-12 lies at the FP64 floor of this system."""
    from .solvers.quasi_static_coupled_solver_2d import quasi_static_coupled_solver_2d
    grid, parts, it, mat, porous, load, dts, cv, H = consolidation_column_dicts(**kw)
    s = quasi_static_coupled_solver_2d(grid, parts, it, mat, porous, load, consolidation_boundary_dofs,
                                       precision=precision, device=device, precond=precond)
    if krylov_rtol is not None:
        s.engine.krylov_rtol = krylov_rtol
    elif precision == "fp64":
        s.engine.krylov_rtol = 1e-10
    top = s.x_particles[:, 1] > grid["end_y"] - grid["dx"] / parts["PPD"]
    s.particle_pressure_boundary_flag_array[:] = top
    s.particle_traction_flag_array[:] = top
    return s, dts, cv, H


# ---------------------------------------------------------------- 3D u-p indentation
def indentation_3d_dicts(block_cells=(80, 80, 48), grid_cells=(96, 96, 64), dx=0.02, PPD=2, E=1e7, nu=0.3,
                         material="Drucker-Prager", cohesion=5e3, friction_angle=30.0, dilation_angle=0.0,
                         permeability=1e-12, viscosity=1e-3, porosity=0.5, indenter=0.4, depth=0.1, n_steps=50,
                         dt=0.1, n_iter=10, tol=1e-9, penalty=None):
    """Constructor dictionaries of the quarter-symmetric indentation of
    problems/3D_indentation/3d_indentation_coupled_cpGIMP.py:11-88 at a given
    size: a block of block_cells cells starting one cell in from the x and y
    symmetry planes and on the base, a rigid square indenter of side
    `indenter` on the block's corner pushed `depth` over n_steps load steps,
    with the reference's penalty-to-modulus ratio of 1 by default."""
    nx, ny, nz = grid_cells
    sx, sy, sz = dx, dx, 0.0
    ex, ey, ez = sx + block_cells[0] * dx, sy + block_cells[1] * dx, sz + block_cells[2] * dx
    grid = dict(n_grid_x=nx, n_grid_y=ny, n_grid_z=nz, max_x=nx * dx, dx=dx, max_y=ny * dx, dy=dx, max_z=nz * dx,
                dz=dx, start_x=sx, end_x=ex, start_y=sy, end_y=ey, start_z=sz, end_z=ez, domain_min_x=sx,
                domain_max_x=ex, domain_min_y=sy, domain_max_y=ey, domain_min_z=sz, domain_max_z=nz * dx)
    n = block_cells[0] * block_cells[1] * block_cells[2] * PPD ** 3
    parts = dict(n_particles=n, PPD=PPD, p_vol=(dx / PPD) ** 3, p_rho=2.0)
    it = dict(n_iter=n_iter, tol=tol, solver_name="scipy", dt=dt)
    mat = dict(youngs_modulus=E, poisson_ratio=nu, material_name=material)
    if material == "Drucker-Prager":
        mat.update(friction_angle=friction_angle, dilation_angle=dilation_angle, cohesion=cohesion, shape_factor=0.0,
                   tension_cutoff=False)
    porous = dict(phi_initial=porosity, mobility_constant=permeability / viscosity)
    load = dict(gravity_mag=0.0, traction_value_x=0.0, traction_value_y=0.0, traction_value_z=0.0,
                point_load_value_x=0.0, point_load_value_y=0.0, point_load_value_z=0.0,
                footing_region_min_x=sx, footing_region_max_x=sx + indenter, footing_region_min_y=sy,
                footing_region_max_y=sy + indenter, footing_initial_height=ez - dx / PPD,
                footing_incr_disp=-depth / n_steps, penalty_factor=E if penalty is None else penalty)
    return grid, parts, it, mat, porous, load


def indentation_boundary_dofs(tid, boundary_flag_array, n_grid_x, n_grid_y, n_nodes, dx, dy, end_x, end_y):
    """set_boundary_dofs of 3d_indentation_coupled_cpGIMP.py:126-153 on index
    tensors: rollers on the symmetry planes and the far walls, fixed base."""
    ix, iy, iz = tid
    dof_x = ix + iy * (n_grid_x + 1) + iz * ((n_grid_x + 1) * (n_grid_y + 1))
    boundary_flag_array[dof_x[(ix <= 1) | ((ix + 0.5) * dx > end_x)]] = True
    boundary_flag_array[(dof_x + n_nodes)[(iy <= 1) | ((iy + 0.5) * dy > end_y)]] = True
    boundary_flag_array[(dof_x + 2 * n_nodes)[iz <= 0]] = True


def indentation_3d(precision="fp64", device=None, precond="mg", **kw):
    """The 3D coupled u-p indentation (keywords of indentation_3d_dicts),
    drained top surface (set_pressure_boundary of the reference script)."""
    from .solvers.quasi_static_coupled_solver_3d import quasi_static_coupled_solver_3d
    grid, parts, it, mat, porous, load = indentation_3d_dicts(**kw)
    s = quasi_static_coupled_solver_3d(grid, parts, it, mat, porous, load, indentation_boundary_dofs,
                                       precision=precision, device=device, precond=precond)
    s.particle_pressure_boundary_flag_array[:] = s.x_particles[:, 2] > grid["end_z"] - grid["dz"] / parts["PPD"]
    return s
