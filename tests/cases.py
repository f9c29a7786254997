"""Problem builders shared by the oracle and the GPU solvers.

Each case returns the reference-style constructor dicts (the API of the
solver classes) plus the boundary-condition setup, so the same problem can be
run through geowarp_b200's drop-in solvers and through the CPU oracle.
"""
import math

import numpy as np

from oracle.mpm import OracleEngine, init_particles_rectangle_2d, init_particles_rectangle_3d


# ---------------------------------------------------------------- 2D solid: bar under self-weight
def bar_dicts(material="Hencky elasticity", height=12.5, E=10.0, nu=0.0, rho=0.08, g=10.0, kappa=5.0,
              n_iter=10, tol=1e-8, extra_mat=None):
    """Reference bar (problems/bar_compaction/bar_compaction_cpGIMP.py:12-61) with a chosen height."""
    n_grid_x = 6
    max_x = 4.6875
    dx = max_x / n_grid_x
    n_cells_y = int(round(height / dx))
    n_grid_y = n_cells_y + 2
    start_x, end_x = dx, 2 * dx
    start_y, end_y = dx, dx + height
    grid = dict(n_grid_x=n_grid_x, n_grid_y=n_grid_y, max_x=max_x, dx=dx, start_x=start_x, end_x=end_x,
                start_y=start_y, end_y=end_y, domain_min_x=start_x, domain_max_x=end_x, domain_min_y=start_y,
                domain_max_y=end_y)
    PPD = 2
    parts = dict(n_particles=4 * n_cells_y, PPD=PPD, p_vol=(dx / PPD) ** 2, p_rho=rho)
    it = dict(n_iter=n_iter, tol=tol, solver_name="scipy")
    mat = dict(youngs_modulus=E, poisson_ratio=nu, material_name=material, kappa=kappa)
    if extra_mat:
        mat.update(extra_mat)
    load = dict(gravity_mag=g, traction_value_x=0.0, traction_value_y=0.0, point_load_value_x=0.0,
                point_load_value_y=0.0)
    return grid, parts, it, mat, load


def bar_boundary(boundary, n_grid_x, n_grid_y):
    """set_boundary_dofs of the bar script (bar_compaction_cpGIMP.py:93-107), NumPy/torch form."""
    nn = (n_grid_x + 1) * (n_grid_y + 1)
    ix = np.tile(np.arange(n_grid_x + 1), n_grid_y + 1)
    iy = np.repeat(np.arange(n_grid_y + 1), n_grid_x + 1)
    dof = ix + iy * (n_grid_x + 1)
    mx = (ix <= 1) | (ix >= 2)
    my = iy <= 1
    bx = dof[mx]
    by = dof[my] + nn
    boundary[bx] = True
    boundary[by] = True


def oracle_solid2d(grid, parts, it, mat, load):
    dx = grid["dx"]
    x = init_particles_rectangle_2d(grid["start_x"], grid["start_y"], grid["end_x"], grid["end_y"], dx,
                                    grid["n_grid_x"], grid["n_grid_y"], parts["PPD"], parts["n_particles"])
    og = dict(n_grid=(grid["n_grid_x"], grid["n_grid_y"]), h=(dx, dx), h_nodes=(dx, dx),
              domain_min=(grid["domain_min_x"], grid["domain_min_y"]),
              domain_max=(grid["domain_max_x"], grid["domain_max_y"]))
    E_field = mat.get("youngs_modulus_field")
    return OracleEngine("solid2d", og, x, parts["p_vol"], parts["p_rho"], parts["PPD"], mat, load,
                        lp0=dx / parts["PPD"] / 2.0 - 1e-6, n_iter=it["n_iter"], tol=it["tol"], E_field=E_field)


# ---------------------------------------------------------------- 2D solid: DP strip footing (small)
def footing_dicts(nx=16, ny=8, dx=0.05, E=2e7, nu=0.3, c=1e4, phi=30.0, psi=0.0, width=0.2, total_disp=0.02,
                  n_steps=10, penalty=1000.0, rho=2000.0, g=0.0, n_iter=15, tol=1e-6, stable=False, geostatic=False):
    """Plane-strain rigid strip footing on Drucker-Prager soil: a soil block of
    nx x ny cells (2x2 particles per cell) in an (nx+4) x (ny+4) grid, rollers
    on the sides, fixed base, penalty footing of the given width centred on the
    top surface, displacement-controlled over n_steps.  geostatic: self-weight
    g = 9.81 at full magnitude from the first step (the caller sets the K0
    initial state)."""
    if geostatic:
        g = 9.81
    n_grid_x, n_grid_y = nx + 4, ny + 4
    start_x, start_y = 2 * dx, 2 * dx
    end_x, end_y = start_x + nx * dx, start_y + ny * dx
    grid = dict(n_grid_x=n_grid_x, n_grid_y=n_grid_y, max_x=n_grid_x * dx, dx=dx, start_x=start_x, end_x=end_x,
                start_y=start_y, end_y=end_y, domain_min_x=start_x, domain_max_x=end_x, domain_min_y=start_y,
                domain_max_y=end_y)
    PPD = 2
    parts = dict(n_particles=nx * ny * PPD * PPD, PPD=PPD, p_vol=(dx / PPD) ** 2, p_rho=rho)
    it = dict(n_iter=n_iter, tol=tol, solver_name="warp")
    mat = dict(youngs_modulus=E, poisson_ratio=nu, material_name="Drucker-Prager", friction_angle=phi,
               dilation_angle=psi, cohesion=c, shape_factor=0.0, tension_cutoff=False)
    xc = 0.5 * (start_x + end_x)
    load = dict(gravity_mag=g, traction_value_x=0.0, traction_value_y=0.0, point_load_value_x=0.0,
                point_load_value_y=0.0, footing_region_min_x=xc - width / 2, footing_region_max_x=xc + width / 2,
                footing_initial_height=end_y - dx / (2 * PPD) if stable else end_y - dx / PPD,
                footing_incr_disp=-total_disp / n_steps, penalty_factor=penalty, footing_penalty_stable=stable,
                gravity_ramp=not geostatic)
    return grid, parts, it, mat, load


def footing_boundary(boundary, grid):
    """Rollers on the side walls (x fixed) and a fixed base (x, y fixed)."""
    nx, ny, dx = grid["n_grid_x"], grid["n_grid_y"], grid["dx"]
    nn = (nx + 1) * (ny + 1)
    ix = np.tile(np.arange(nx + 1), ny + 1)
    iy = np.repeat(np.arange(ny + 1), nx + 1)
    dof = ix + iy * (nx + 1)
    i0 = int(round(grid["start_x"] / dx))
    i1 = int(round(grid["end_x"] / dx))
    j0 = int(round(grid["start_y"] / dx))
    side = (ix <= i0) | (ix >= i1)
    base = iy <= j0
    boundary[dof[side | base]] = True
    boundary[dof[base] + nn] = True


# ---------------------------------------------------------------- 2D u-p: consolidation column (small)
def terzaghi_dicts(n_cells_y=20, dx=0.1, E=1500.0, nu=0.25, mobility=1e-6, phi0=0.5, traction=-1.0, dt=100.0,
                   n_iter=10, tol=1e-8, material="Neo-Hookean"):
    """problems/consolidation/terzaghi_cpGIMP.py:12-73 with a shorter column."""
    n_grid_x = 6
    max_x = n_grid_x * dx
    n_grid_y = n_cells_y + 2
    max_y = n_grid_y * dx
    start_x, end_x = dx, 2 * dx
    start_y, end_y = 0.0, n_cells_y * dx
    grid = dict(n_grid_x=n_grid_x, n_grid_y=n_grid_y, max_x=max_x, dx=dx, max_y=max_y, dy=max_y / n_grid_y,
                start_x=start_x, end_x=end_x, start_y=start_y, end_y=end_y, domain_min_x=start_x,
                domain_max_x=end_x, domain_min_y=start_y, domain_max_y=max_y)
    PPD = 2
    parts = dict(n_particles=4 * n_cells_y, PPD=PPD, p_vol=(dx / PPD) ** 2, p_rho=1.0)
    it = dict(n_iter=n_iter, tol=tol, solver_name="scipy", dt=dt)
    mat = dict(youngs_modulus=E, poisson_ratio=nu, material_name=material)
    porous = dict(phi_initial=phi0, mobility_constant=mobility)
    load = dict(gravity_mag=0.0, traction_value_x=0.0, traction_value_y=traction, point_load_value_x=0.0,
                point_load_value_y=0.0)
    return grid, parts, it, mat, porous, load


def terzaghi_boundary_np(boundary, n_grid_x, n_grid_y):
    """set_boundary_dofs of terzaghi_cpGIMP.py:104-119."""
    nn = (n_grid_x + 1) * (n_grid_y + 1)
    ix = np.tile(np.arange(n_grid_x + 1), n_grid_y + 1)
    iy = np.repeat(np.arange(n_grid_y + 1), n_grid_x + 1)
    dof = ix + iy * (n_grid_x + 1)
    boundary[dof[(ix <= 1) | (ix >= 2)]] = True
    boundary[dof[iy <= 0] + nn] = True


def terzaghi_boundary_kernel(tid, boundary_flag_array, n_grid_x, n_nodes):
    """The same kernel in geowarp_b200.launch form (index tensors first)."""
    node_idx, node_idy = tid
    dof_x = node_idx + node_idy * (n_grid_x + 1)
    dof_y = dof_x + n_nodes
    boundary_flag_array[dof_x[(node_idx <= 1) | (node_idx >= 2)]] = True
    boundary_flag_array[dof_y[node_idy <= 0]] = True


def top_flags(x, end_y, dx, PPD):
    """set_traction_boundary / set_pressure_boundary (terzaghi_cpGIMP.py:127-149)."""
    return x[:, 1] > end_y - dx / PPD


def oracle_coupled2d(grid, parts, it, mat, porous, load):
    dx = grid["dx"]
    x = init_particles_rectangle_2d(grid["start_x"], grid["start_y"], grid["end_x"], grid["end_y"], dx,
                                    grid["n_grid_x"], grid["n_grid_y"], parts["PPD"], parts["n_particles"])
    og = dict(n_grid=(grid["n_grid_x"], grid["n_grid_y"]), h=(dx, dx), h_nodes=(dx, grid["dy"]),
              domain_min=(grid["domain_min_x"], grid["domain_min_y"]),
              domain_max=(grid["domain_max_x"], grid["domain_max_y"]))
    return OracleEngine("coupled2d", og, x, parts["p_vol"], parts["p_rho"], parts["PPD"], mat, load,
                        lp0=dx / parts["PPD"] / 2.0 - 1e-6, n_iter=it["n_iter"], tol=it["tol"], dt=it["dt"],
                        phi_initial=porous["phi_initial"], mobility=porous["mobility_constant"],
                        mobility_law=porous.get("mobility_law", "constant"),
                        p2g_projection=porous.get("p2g_projection", "consistent"))


# ---------------------------------------------------------------- 3D u-p: indentation (small)
def indentation_dicts(n=4, dx=0.25, PPD=2, E=1e3, nu=0.3, mobility=1e-8, dt=0.1, n_iter=10, tol=1e-9,
                      material="Neo-Hookean", incr=-0.02, penalty=1000.0):
    """problems/3D_indentation/3d_indentation_coupled_cpGIMP.py:11-88 scaled
    down to an n x n x n cell block."""
    n_grid = n + 2
    max_x = n_grid * dx
    start_x = start_y = dx
    start_z = 0.0
    end_x, end_y, end_z = start_x + n * dx, start_y + n * dx, start_z + n * dx
    grid = dict(n_grid_x=n_grid, n_grid_y=n_grid, n_grid_z=n_grid, max_x=max_x, dx=dx, max_y=max_x, dy=dx,
                max_z=max_x, dz=dx, start_x=start_x, end_x=end_x, start_y=start_y, end_y=end_y, start_z=start_z,
                end_z=end_z, domain_min_x=start_x, domain_max_x=end_x, domain_min_y=start_y, domain_max_y=end_y,
                domain_min_z=start_z, domain_max_z=max_x)
    parts = dict(n_particles=n ** 3 * PPD ** 3, PPD=PPD, p_vol=(dx / PPD) ** 3, p_rho=2.0)
    it = dict(n_iter=n_iter, tol=tol, solver_name="scipy", dt=dt)
    mat = dict(youngs_modulus=E, poisson_ratio=nu, material_name=material)
    porous = dict(phi_initial=0.5, mobility_constant=mobility)
    load = dict(gravity_mag=0.0, traction_value_x=0.0, traction_value_y=0.0, traction_value_z=0.0,
                point_load_value_x=0.0, point_load_value_y=0.0, point_load_value_z=0.0,
                footing_region_min_x=start_x, footing_region_max_x=start_x + 2 * dx, footing_region_min_y=start_y,
                footing_region_max_y=start_y + 2 * dx, footing_initial_height=end_z - dx / PPD,
                footing_incr_disp=incr, penalty_factor=penalty)
    return grid, parts, it, mat, porous, load


def indentation_boundary_np(boundary, grid):
    """set_boundary_dofs of 3d_indentation_coupled_cpGIMP.py:126-153."""
    nx, ny, nz = grid["n_grid_x"], grid["n_grid_y"], grid["n_grid_z"]
    nn = (nx + 1) * (ny + 1) * (nz + 1)
    iz, iy, ix = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    ix, iy, iz = ix.ravel(), iy.ravel(), iz.ravel()
    dof = ix + iy * (nx + 1) + iz * (nx + 1) * (ny + 1)
    boundary[dof[(ix <= 1) | ((ix + 0.5) * grid["dx"] > grid["end_x"])]] = True
    boundary[dof[(iy <= 1) | ((iy + 0.5) * grid["dy"] > grid["end_y"])] + nn] = True
    boundary[dof[iz <= 0] + 2 * nn] = True


def indentation_boundary_kernel(tid, boundary_flag_array, n_grid_x, n_grid_y, n_nodes, dx, dy, end_x, end_y):
    node_idx, node_idy, node_idz = tid
    dof_x = node_idx + node_idy * (n_grid_x + 1) + node_idz * ((n_grid_x + 1) * (n_grid_y + 1))
    boundary_flag_array[dof_x[(node_idx <= 1) | ((node_idx + 0.5) * dx > end_x)]] = True
    boundary_flag_array[(dof_x + n_nodes)[(node_idy <= 1) | ((node_idy + 0.5) * dy > end_y)]] = True
    boundary_flag_array[(dof_x + 2 * n_nodes)[node_idz <= 0]] = True


def oracle_coupled3d(grid, parts, it, mat, porous, load):
    dx = grid["dx"]
    x = init_particles_rectangle_3d(grid["start_x"], grid["start_y"], grid["start_z"], grid["end_x"], grid["end_y"],
                                    grid["end_z"], dx, grid["n_grid_x"], grid["n_grid_y"], grid["n_grid_z"],
                                    parts["PPD"], parts["n_particles"])
    og = dict(n_grid=(grid["n_grid_x"], grid["n_grid_y"], grid["n_grid_z"]), h=(dx, grid["dy"], grid["dz"]),
              h_nodes=(dx, grid["dy"], grid["dz"]),
              domain_min=(grid["domain_min_x"], grid["domain_min_y"], grid["domain_min_z"]),
              domain_max=(grid["domain_max_x"], grid["domain_max_y"], grid["domain_max_z"]))
    return OracleEngine("coupled3d", og, x, parts["p_vol"], parts["p_rho"], parts["PPD"], mat, load,
                        lp0=dx / parts["PPD"] / 2.0, n_iter=it["n_iter"], tol=it["tol"], dt=it["dt"],
                        phi_initial=porous["phi_initial"], mobility=porous["mobility_constant"])


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / den)
