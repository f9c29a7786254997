"""Drop-in 2D u-p coupled quasi-static implicit cpGIMP solver.

Mirrors solvers/quasi_static_coupled_solver_2d.py:45-313: same dicts, the
set_boundary_dofs callback invoked every step over the (nx+1, ny+1) node
lattice with inputs (boundary_flag_array, n_grid_x, n_nodes), consistent-mass
projection of the particle pressure (host pyamg in the reference, a GPU CG
here), Newton on (ux, uy, p), G2P.  set_boundary_dofs follows the calling
convention of geowarp_b200.launch (index tensors first, then the inputs).

Extensions: 'Linear elasticity' and 'Drucker-Prager' skeletons next to the
reference's 'Neo-Hookean'; solver.dt may be changed between steps (log-spaced
time stepping).
"""
import numpy as np
import torch

from ..engine import Engine, material_struct
from ..launch import launch
from ..mpm.mpm_utils import init_particles_rectangle_2d
from .quasi_static_solver_2d import DofStruct

SUPPORTED = ("Neo-Hookean", "Linear elasticity", "Hencky elasticity", "Drucker-Prager")


class quasi_static_coupled_solver_2d:
    def __init__(self, background_grid_dict, particles_dict, iteration_dict, material_dict, porous_media_dict,
                 load_dict, set_boundary_dofs, precision="fp64", device=None, precond="block"):
        g = background_grid_dict
        self.n_grid_x = g["n_grid_x"]
        self.n_grid_y = g["n_grid_y"]
        self.n_nodes = (self.n_grid_x + 1) * (self.n_grid_y + 1)
        self.n_matrix_size = 3 * self.n_nodes
        self.max_x, self.dx = g["max_x"], g["dx"]
        self.max_y, self.dy = g["max_y"], g["dy"]
        self.inv_dx, self.inv_dy = 1.0 / self.dx, 1.0 / self.dy
        self.start_x, self.end_x = g["start_x"], g["end_x"]
        self.start_y, self.end_y = g["start_y"], g["end_y"]
        self.domain_min_x, self.domain_max_x = g["domain_min_x"], g["domain_max_x"]
        self.domain_min_y, self.domain_max_y = g["domain_min_y"], g["domain_max_y"]

        self.n_particles = particles_dict["n_particles"]
        self.PPD = particles_dict["PPD"]
        self.p_vol = particles_dict["p_vol"]
        self.p_rho = particles_dict["p_rho"]
        self.p_mass = self.p_vol * self.p_rho
        self.GIMP_lp_initial = self.dx / self.PPD / 2.0 - 1e-6

        self.n_iter = iteration_dict["n_iter"]
        self.tol = iteration_dict["tol"]
        self.solver_name = iteration_dict.get("solver_name", "scipy")
        self.dt = iteration_dict["dt"]

        self.youngs_modulus = material_dict["youngs_modulus"]
        self.poisson_ratio = material_dict["poisson_ratio"]
        nu = self.poisson_ratio
        self.lame_lambda = self.youngs_modulus * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
        self.lame_mu = self.youngs_modulus / (2.0 * (1.0 + nu))
        self.material_name = material_dict["material_name"]
        if self.material_name not in SUPPORTED:
            raise ValueError(f"Unimplemented material model: {self.material_name}")
        self._mat = material_struct(material_dict)

        self.phi_initial = porous_media_dict["phi_initial"]
        self.mobility_constant = porous_media_dict["mobility_constant"]
        # extensions from the reference's large-deformation consolidation script
        # (problems/consolidation/large_consolidation_cpGIMP_everything_in_one_script.py):
        # the J-dependent mobility of :330-338 ("Uzuoka-Borja") and the lumped
        # pressure projection of :292-310 ("lumped"); the defaults keep the solver
        # class's own behaviour (constant mobility, consistent-mass projection)
        self.mobility_law = porous_media_dict.get("mobility_law", "constant")
        self.p2g_projection = porous_media_dict.get("p2g_projection", "consistent")
        if self.p2g_projection not in ("consistent", "lumped"):
            raise ValueError(f"unknown pressure projection {self.p2g_projection!r}")

        self.gravity_mag = load_dict["gravity_mag"]
        self.traction_value_x = load_dict.get("traction_value_x", 0.0)
        self.traction_value_y = load_dict.get("traction_value_y", 0.0)
        self.point_load_value_x = load_dict.get("point_load_value_x", 0.0)
        self.point_load_value_y = load_dict.get("point_load_value_y", 0.0)
        self.set_boundary_dofs = set_boundary_dofs

        x = init_particles_rectangle_2d(self.start_x, self.start_y, self.end_x, self.end_y, self.dx, self.n_grid_x,
                                        self.n_grid_y, self.PPD, self.n_particles)
        # shape functions use dx on both axes (mpm/gimp.py:26-31); nodal
        # positions for pressure BCs use (dx, dy) (mpm/mpm_utils.py:230)
        self.engine = Engine("coupled2d", (self.n_grid_x, self.n_grid_y), (self.dx, self.dx), (self.dx, self.dy),
                             (self.domain_min_x, self.domain_min_y), (self.domain_max_x, self.domain_max_y), x,
                             device=device, precision=precision, precond=precond)
        e = self.engine
        e.lp.fill_(self.GIMP_lp_initial)
        field = material_dict.get("youngs_modulus_field")
        if field is not None:
            e.E = torch.as_tensor(np.asarray(field, dtype=np.float64), device=e.device).contiguous()
        self.dofStruct = DofStruct(e)

    # ------------------------------------------------------------------ public arrays
    x_particles = property(lambda self: self.engine.x)
    x0 = property(lambda self: self.engine.x0)
    deformation_gradient_total_new = property(lambda self: self.engine.F_new)
    deformation_gradient_total_old = property(lambda self: self.engine.F_old)
    left_Cauchy_Green_new = property(lambda self: self.engine.b_new)
    left_Cauchy_Green_old = property(lambda self: self.engine.b_old)
    particle_Cauchy_stress_array = property(lambda self: self.engine.sigma)
    particle_pressure_array = property(lambda self: self.engine.pressure)
    GIMP_lp = property(lambda self: self.engine.lp)
    particle_external_flag_array = property(lambda self: self.engine.ext_flag)
    particle_traction_flag_array = property(lambda self: self.engine.trac_flag)
    particle_pressure_boundary_flag_array = property(lambda self: self.engine.pbc_flag)

    @property
    def new_solution(self):
        return self.engine.node_to_field_major(self.engine.u_new)

    @property
    def old_solution(self):
        return self.engine.node_to_field_major(self.engine.u_old)

    def _set_step_params(self):
        self.engine.step_params = dict(
            gravity_mag=self.gravity_mag, point_load=(self.point_load_value_x, self.point_load_value_y, 0.0),
            traction=(self.traction_value_x, self.traction_value_y, 0.0), p_vol=self.p_vol, p_rho=self.p_rho,
            PPD=self.PPD, lp0=self.GIMP_lp_initial, dt=self.dt, phi_initial=self.phi_initial,
            mobility=self.mobility_constant, mobility_law=self.mobility_law)

    # ------------------------------------------------------------------ methods
    def reset(self):
        """Solutions, boundary and activation flags := 0 (reference :164-175)."""
        self.engine.reset(clear_boundary=True)

    def newton_iter(self, current_step, total_steps):
        return self.engine.newton(self._mat, current_step, total_steps, self.n_iter, self.tol)

    def advance_one_step(self, current_step, total_steps):
        e = self.engine
        self._set_step_params()
        self.reset()
        if self.set_boundary_dofs is not None:
            launch(self.set_boundary_dofs, (self.n_grid_x + 1, self.n_grid_y + 1),
                   [self.dofStruct.boundary_flag_array, self.n_grid_x, self.n_nodes])
        e.sort_and_activate()
        e.project_pressure(lumped=self.p2g_projection == "lumped")
        e.build_system()
        self.newton_iter(current_step, total_steps)
        e.g2p(current_step, total_steps)
