"""Drop-in 3D u-p coupled quasi-static implicit cpGIMP solver with the
penalty indenter and the indentation-force inverse hooks.

Mirrors solvers/quasi_static_coupled_solver_3d.py:56-420: same dicts, the
set_boundary_dofs callback over the (nx+1, ny+1, nz+1) lattice with inputs
(boundary_flag_array, n_grid_x, n_grid_y, n_nodes, dx, dy, end_x, end_y),
consistent-mass projection (Warp BiCGSTAB there, a GPU CG here), Newton on
(ux, uy, uz, p), G2P inside newton_iter, the per-step indentation force list,
the loss (F/(|d|N) - 13567.27337196)^2 (:45-52) and E_grad, the derivative of
that loss with respect to Young's modulus at the last Newton iterate of the
last step with the state held fixed (the quantity of :323-325).  Scripts may
mutate dz / inv_dz between steps (moving mesh) and call reinit_everything,
reset_grid and reset_youngs_modulus exactly as the reference allows.
"""
import numpy as np
import torch

from ..engine import Engine, material_struct
from ..launch import launch
from ..mpm.mpm_utils import init_particles_rectangle_3d
from .quasi_static_solver_2d import DofStruct

LOSS_TARGET = 13567.27337196  # solvers/quasi_static_coupled_solver_3d.py:52
SUPPORTED = ("Neo-Hookean", "Linear elasticity", "Hencky elasticity", "Drucker-Prager")


class quasi_static_coupled_solver_3d:
    def __init__(self, background_grid_dict, particles_dict, iteration_dict, material_dict, porous_media_dict,
                 load_dict, set_boundary_dofs, precision="fp64", device=None, precond="block", n_force_slots=25):
        g = background_grid_dict
        self.n_grid_x, self.n_grid_y, self.n_grid_z = g["n_grid_x"], g["n_grid_y"], g["n_grid_z"]
        self.n_nodes = (self.n_grid_x + 1) * (self.n_grid_y + 1) * (self.n_grid_z + 1)
        self.n_matrix_size = 4 * self.n_nodes
        self.max_x, self.dx = g["max_x"], g["dx"]
        self.max_y, self.dy = g["max_y"], g["dy"]
        self.max_z, self.dz = g["max_z"], g["dz"]
        self.inv_dx, self.inv_dy, self.inv_dz = 1.0 / self.dx, 1.0 / self.dy, 1.0 / self.dz
        self.start_x, self.end_x = g["start_x"], g["end_x"]
        self.start_y, self.end_y = g["start_y"], g["end_y"]
        self.start_z, self.end_z = g["start_z"], g["end_z"]
        self.domain_min_x, self.domain_max_x = g["domain_min_x"], g["domain_max_x"]
        self.domain_min_y, self.domain_max_y = g["domain_min_y"], g["domain_max_y"]
        self.domain_min_z, self.domain_max_z = g["domain_min_z"], g["domain_max_z"]

        self.n_particles = particles_dict["n_particles"]
        self.PPD = particles_dict["PPD"]
        self.p_vol = particles_dict["p_vol"]
        self.p_rho = particles_dict["p_rho"]
        self.p_mass = self.p_vol * self.p_rho
        self.GIMP_lp_initial = self.dx / self.PPD / 2.0  # no -1e-6 offset in 3D (reference :100)

        self.n_iter = iteration_dict["n_iter"]
        self.tol = iteration_dict["tol"]
        self.solver_name = iteration_dict.get("solver_name", "warp")
        self.dt = iteration_dict["dt"]

        self.material_dict = dict(material_dict)
        self.youngs_modulus = material_dict["youngs_modulus"]
        self.poisson_ratio = material_dict["poisson_ratio"]
        self.material_name = material_dict["material_name"]
        if self.material_name not in SUPPORTED:
            raise ValueError(f"Unimplemented material model: {self.material_name}")
        self.reset_youngs_modulus(self.youngs_modulus)

        self.phi_initial = porous_media_dict["phi_initial"]
        self.mobility_constant = porous_media_dict["mobility_constant"]

        ld = load_dict
        self.gravity_mag = ld["gravity_mag"]
        self.traction_value_x = ld.get("traction_value_x", 0.0)
        self.traction_value_y = ld.get("traction_value_y", 0.0)
        self.traction_value_z = ld.get("traction_value_z", 0.0)
        self.point_load_value_x = ld.get("point_load_value_x", 0.0)
        self.point_load_value_y = ld.get("point_load_value_y", 0.0)
        self.point_load_value_z = ld.get("point_load_value_z", 0.0)
        self.footing_region_min_x = ld["footing_region_min_x"]
        self.footing_region_max_x = ld["footing_region_max_x"]
        self.footing_region_min_y = ld["footing_region_min_y"]
        self.footing_region_max_y = ld["footing_region_max_y"]
        self.footing_initial_height = ld["footing_initial_height"]
        self.footing_incr_disp = ld["footing_incr_disp"]
        self.penalty_factor = ld["penalty_factor"]
        self.set_boundary_dofs = set_boundary_dofs

        x = self._seed()
        self.engine = Engine("coupled3d", (self.n_grid_x, self.n_grid_y, self.n_grid_z), (self.dx, self.dy, self.dz),
                             (self.dx, self.dy, self.dz),
                             (self.domain_min_x, self.domain_min_y, self.domain_min_z),
                             (self.domain_max_x, self.domain_max_y, self.domain_max_z), x,
                             device=device, precision=precision, precond=precond)
        e = self.engine
        e.lp.fill_(self.GIMP_lp_initial)
        e.F_old[:] = torch.tensor([[1.0 + 1e-7, 0, 0], [0, 1.0 - 1e-6, 0], [0, 0, 1.0]], dtype=torch.float64,
                                  device=e.device)
        self.dofStruct = DofStruct(e)
        self.indentation_force_list = np.empty(0)
        self.indentation_force_array = np.zeros(n_force_slots)
        self.indentation_force = np.zeros(1)
        self.loss = np.zeros(1)
        self.E_grad = None

    def _seed(self):
        return init_particles_rectangle_3d(self.start_x, self.start_y, self.start_z, self.end_x, self.end_y,
                                           self.end_z, self.dx, self.n_grid_x, self.n_grid_y, self.n_grid_z,
                                           self.PPD, self.n_particles)

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

    # ------------------------------------------------------------------ inverse-analysis hooks
    def reinit_everything(self):
        """Re-seed particles and reset their state (reference :206-221)."""
        e = self.engine
        e.x.copy_(torch.as_tensor(self._seed(), device=e.device))
        self.E_grad = None
        self.indentation_force_list = np.empty(0)
        e.pressure.zero_()
        ident = torch.tensor([[1.0 + 1e-7, 0, 0], [0, 1.0 - 1e-6, 0], [0, 0, 1.0]], dtype=torch.float64, device=e.device)
        for t in (e.F_new, e.F_old, e.b_new, e.b_old):
            t[:] = ident
        e.lp.fill_(self.GIMP_lp_initial)

    def reset_grid(self, dx, dy, dz):
        self.dx, self.dy, self.dz = dx, dy, dz
        self.inv_dx, self.inv_dy, self.inv_dz = 1.0 / dx, 1.0 / dy, 1.0 / dz

    def reset_youngs_modulus(self, youngs_modulus):
        self.youngs_modulus = youngs_modulus
        nu = self.poisson_ratio
        self.lame_lambda = youngs_modulus * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
        self.lame_mu = youngs_modulus / (2.0 * (1.0 + nu))
        md = dict(self.material_dict)
        md["youngs_modulus"] = youngs_modulus
        self._mat = material_struct(md)

    # ------------------------------------------------------------------ methods
    def _sync_grid(self):
        # scripts mutate dz/inv_dz between steps (moving mesh); the shape
        # functions read the current values (reference passes self.dz each launch)
        e = self.engine
        e.h = (self.dx, self.dy, self.dz)
        e.h_nodes = (self.dx, self.dy, self.dz)

    def _set_step_params(self):
        self.engine.step_params = dict(
            gravity_mag=self.gravity_mag,
            point_load=(self.point_load_value_x, self.point_load_value_y, self.point_load_value_z),
            traction=(self.traction_value_x, self.traction_value_y, self.traction_value_z),
            p_vol=self.p_vol, p_rho=self.p_rho, PPD=self.PPD, lp0=self.GIMP_lp_initial, dt=self.dt,
            phi_initial=self.phi_initial, mobility=self.mobility_constant,
            footing=dict(min=(self.footing_region_min_x, self.footing_region_min_y),
                         max=(self.footing_region_max_x, self.footing_region_max_y),
                         initial_height=self.footing_initial_height, incr_disp=self.footing_incr_disp,
                         penalty_factor=self.penalty_factor))

    def reset(self):
        self.engine.reset(clear_boundary=True)

    def newton_iter(self, current_step, total_steps):
        e = self.engine
        its = e.newton(self._mat, current_step, total_steps, self.n_iter, self.tol)
        force = float(e.force.item())
        self.indentation_force[0] = force
        if 0 <= int(current_step) < self.indentation_force_array.size:
            self.indentation_force_array[:] = 0.0
            self.indentation_force_array[int(current_step)] = force
        scale = abs(self.footing_incr_disp) * total_steps
        self.loss[0] = (force / scale - LOSS_TARGET) ** 2
        if current_step == total_steps - 1:
            # force is linear in E through the penalty stiffness at fixed state
            self.E_grad = np.array([2.0 * (force / scale - LOSS_TARGET) * (force / self.youngs_modulus) / scale])
        e.g2p(current_step, total_steps)
        self.indentation_force_list = np.append(self.indentation_force_list, force)
        return its

    def advance_one_step(self, current_step, total_steps):
        e = self.engine
        self._sync_grid()
        self._set_step_params()
        self.reset()
        if self.set_boundary_dofs is not None:
            launch(self.set_boundary_dofs, (self.n_grid_x + 1, self.n_grid_y + 1, self.n_grid_z + 1),
                   [self.dofStruct.boundary_flag_array, self.n_grid_x, self.n_grid_y, self.n_nodes, self.dx, self.dy,
                    self.end_x, self.end_y])
        e.sort_and_activate()
        e.project_pressure()
        e.build_system()
        self.newton_iter(current_step, total_steps)
