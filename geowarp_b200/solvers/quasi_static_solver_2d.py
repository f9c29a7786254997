"""Drop-in 2D solid quasi-static implicit cpGIMP solver.

Mirrors solvers/quasi_static_solver_2d.py:45-258 of the reference: same
constructor dicts, same methods (reset, newton_iter, advance_one_step), same
public arrays (x_particles, x0, particle_Cauchy_stress_array,
particle_external_flag_array, dofStruct.boundary_flag_array, ...), now torch
tensors on the GPU.  The step runs on the CUDA kernels of libgeowarp_b200.so:
the Jacobian is assembled element by element from exact particle tangents
instead of 50 coloured reverse-mode sweeps, and the linear system is solved by
the GPU Krylov solver for every solver_name ('warp', 'scipy', 'pyamg').

Extensions (documented, off by default): material_name 'Neo-Hookean',
'Linear elasticity', 'Drucker-Prager', 'NorSand'; a penalty strip footing
(load_dict keys footing_region_min_x/max_x, footing_initial_height,
footing_incr_disp, penalty_factor), the 2D restatement of the reference's 3D
penalty indenter (mpm/mpm_utils.py:1234-1248); per-particle Young's modulus
via material_dict['youngs_modulus_field']; precision='mixed'.
"""
import numpy as np
import torch

from ..engine import Engine, material_struct
from ..mpm.mpm_utils import init_particles_rectangle_2d

SUPPORTED = ("Hencky elasticity", "J2", "Neo-Hookean", "Linear elasticity", "Drucker-Prager", "NorSand")


class DofStruct:
    """activate_flag_array / boundary_flag_array in the reference's field-major
    DOF order (x-DOF = node id, y-DOF = node id + n_nodes)."""

    def __init__(self, engine):
        self._e = engine

    @property
    def boundary_flag_array(self):
        return self._e.boundary

    @property
    def activate_flag_array(self):
        return self._e.node_active.bool().repeat(self._e.nf)


class quasi_static_solver_2d:
    def __init__(self, background_grid_dict, particles_dict, iteration_dict, material_dict, load_dict,
                 precision="fp64", device=None, precond="mg", x_particles=None):
        """x_particles (extension): particle positions [n_particles, 2] to use
        instead of the regular seeding of the start/end box (e.g. several
        separate blocks in one grid)."""
        g = background_grid_dict
        self.n_grid_x = g["n_grid_x"]
        self.n_grid_y = g["n_grid_y"]
        self.n_nodes = (self.n_grid_x + 1) * (self.n_grid_y + 1)
        self.n_matrix_size = 2 * self.n_nodes
        self.max_x = g["max_x"]
        self.dx = g["dx"]
        self.inv_dx = 1.0 / self.dx
        self.start_x, self.end_x = g["start_x"], g["end_x"]
        self.start_y, self.end_y = g["start_y"], g["end_y"]
        self.domain_min_x, self.domain_max_x = g["domain_min_x"], g["domain_max_x"]
        self.domain_min_y, self.domain_max_y = g["domain_min_y"], g["domain_max_y"]

        self.n_particles = particles_dict["n_particles"]
        self.PPD = particles_dict["PPD"]
        self.p_vol = particles_dict["p_vol"]
        self.p_rho = particles_dict["p_rho"]
        self.GIMP_lp_initial = self.dx / self.PPD / 2.0 - 1e-6

        self.n_iter = iteration_dict["n_iter"]
        self.tol = iteration_dict["tol"]
        self.solver_name = iteration_dict.get("solver_name", "warp")

        self.material_dict = dict(material_dict)
        self.youngs_modulus = material_dict["youngs_modulus"]
        self.poisson_ratio = material_dict["poisson_ratio"]
        nu = self.poisson_ratio
        self.lame_lambda = self.youngs_modulus * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
        self.lame_mu = self.youngs_modulus / (2.0 * (1.0 + nu))
        self.material_name = material_dict["material_name"]
        if self.material_name not in SUPPORTED:
            raise ValueError(f"Unimplemented material model: {self.material_name}")
        if self.material_name == "J2":
            self.kappa = material_dict["kappa"]
        self._mat = material_struct(material_dict)

        self.gravity_mag = load_dict["gravity_mag"]
        self.traction_value_x = load_dict.get("traction_value_x", 0.0)
        self.traction_value_y = load_dict.get("traction_value_y", 0.0)
        self.point_load_value_x = load_dict.get("point_load_value_x", 0.0)
        self.point_load_value_y = load_dict.get("point_load_value_y", 0.0)
        self.load_dict = dict(load_dict)

        if x_particles is None:
            x = init_particles_rectangle_2d(self.start_x, self.start_y, self.end_x, self.end_y, self.dx, self.n_grid_x,
                                            self.n_grid_y, self.PPD, self.n_particles)
        else:
            x = np.asarray(x_particles, dtype=np.float64).reshape(self.n_particles, 2)
        self.engine = Engine("solid2d", (self.n_grid_x, self.n_grid_y), (self.dx, self.dx), (self.dx, self.dx),
                             (self.domain_min_x, self.domain_min_y), (self.domain_max_x, self.domain_max_y), x,
                             device=device, precision=precision, precond=precond)
        e = self.engine
        e.lp.fill_(self.GIMP_lp_initial)
        field = material_dict.get("youngs_modulus_field")
        if field is not None:
            e.E = torch.as_tensor(np.asarray(field, dtype=np.float64), device=e.device).contiguous()
        self.dofStruct = DofStruct(e)
        self._set_step_params()

    # ------------------------------------------------------------------ public arrays
    @property
    def x_particles(self):
        return self.engine.x

    @property
    def x0(self):
        return self.engine.x0

    @property
    def deformation_gradient_total_new(self):
        return self.engine.F_new

    @property
    def deformation_gradient_total_old(self):
        return self.engine.F_old

    @property
    def left_Cauchy_Green_new(self):
        return self.engine.b_new

    @property
    def left_Cauchy_Green_old(self):
        return self.engine.b_old

    @property
    def particle_Cauchy_stress_array(self):
        return self.engine.sigma

    @property
    def GIMP_lp(self):
        return self.engine.lp

    @property
    def particle_external_flag_array(self):
        return self.engine.ext_flag

    @property
    def increment_solution(self):
        """Field-major nodal increment (reference layout)."""
        return self.engine.node_to_field_major(self.engine.u_new)

    @property
    def rhs(self):
        """Field-major residual of the last assembled Newton iterate."""
        return self.engine.rows_to_field_major(self.engine._R)

    def _set_step_params(self):
        ld = self.load_dict
        sp = dict(gravity_mag=self.gravity_mag, point_load=(self.point_load_value_x, self.point_load_value_y, 0.0),
                  traction=(0.0, 0.0, 0.0), p_vol=self.p_vol, p_rho=self.p_rho, PPD=self.PPD,
                  lp0=self.GIMP_lp_initial, gravity_ramp=bool(ld.get("gravity_ramp", True)))
        if "penalty_factor" in ld:
            sp["footing"] = dict(min=(ld["footing_region_min_x"], 0.0), max=(ld["footing_region_max_x"], 0.0),
                                 initial_height=ld["footing_initial_height"], incr_disp=ld["footing_incr_disp"],
                                 penalty_factor=ld["penalty_factor"],
                                 stable=bool(ld.get("footing_penalty_stable", False)))
        self.engine.step_params = sp

    @property
    def footing_force(self):
        return float(self.engine.force.item())

    # ------------------------------------------------------------------ methods
    def reset(self):
        """increment := 0, activation := 0; Dirichlet flags persist (reference :144-147)."""
        self.engine.reset(clear_boundary=False)

    def newton_iter(self, current_step, total_steps):
        return self.engine.newton(self._mat, current_step, total_steps, self.n_iter, self.tol)

    def advance_one_step(self, current_step, total_steps):
        e = self.engine
        self._set_step_params()
        self.reset()
        e.sort_and_activate()
        e.build_system()
        self.newton_iter(current_step, total_steps)
        e.g2p(current_step, total_steps)
