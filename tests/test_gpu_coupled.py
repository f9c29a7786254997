"""GPU parity: u-p coupled solvers (2D consolidation column, 3D indentation) against the CPU oracle."""
import numpy as np
import pytest
import torch

import cases
from cases import rel_err

pytestmark = pytest.mark.gpu


def test_terzaghi_matches_oracle(cuda):
    from geowarp_b200.solvers import quasi_static_coupled_solver_2d
    grid, parts, it, mat, porous, load = cases.terzaghi_dicts(n_cells_y=12)
    s = quasi_static_coupled_solver_2d(grid, parts, it, mat, porous, load, cases.terzaghi_boundary_kernel)
    top = cases.top_flags(s.x_particles, grid["end_y"], grid["dx"], parts["PPD"])
    s.particle_pressure_boundary_flag_array[:] = top
    s.particle_traction_flag_array[:] = top
    o = cases.oracle_coupled2d(grid, parts, it, mat, porous, load)
    topn = cases.top_flags(o.x, grid["end_y"], grid["dx"], parts["PPD"])
    o.pbc_flag[:] = topn
    o.trac_flag[:] = topn
    bnd = lambda b: cases.terzaghi_boundary_np(b, grid["n_grid_x"], grid["n_grid_y"])
    for k in range(4):
        s.advance_one_step(k, 600)
        o.advance_one_step(k, 600, set_boundary=bnd)
    assert rel_err(s.particle_pressure_array.cpu().numpy(), o.pressure) < 1e-9
    assert rel_err(s.x_particles.cpu().numpy() - o.x0, o.x - o.x0) < 1e-9
    assert rel_err(s.particle_Cauchy_stress_array.cpu().numpy(), o.sigma) < 1e-9
    assert np.array_equal(s.dofStruct.boundary_flag_array.cpu().numpy(), o.boundary)


@pytest.mark.parametrize("material", ["Neo-Hookean"])
def test_indentation3d_matches_oracle(cuda, material):
    from geowarp_b200.solvers import quasi_static_coupled_solver_3d
    grid, parts, it, mat, porous, load = cases.indentation_dicts(n=4, material=material)
    s = quasi_static_coupled_solver_3d(grid, parts, it, mat, porous, load, cases.indentation_boundary_kernel)
    pb = s.x_particles[:, 2] > grid["end_z"] - grid["dz"] / parts["PPD"]
    s.particle_pressure_boundary_flag_array[:] = pb
    o = cases.oracle_coupled3d(grid, parts, it, mat, porous, load)
    o.pbc_flag[:] = o.x[:, 2] > grid["end_z"] - grid["dz"] / parts["PPD"]
    bnd = lambda b: cases.indentation_boundary_np(b, grid)
    for k in range(2):
        s.advance_one_step(k, 25)
        o.advance_one_step(k, 25, set_boundary=bnd)
    assert rel_err(s.x_particles.cpu().numpy() - o.x0, o.x - o.x0) < 1e-9
    assert rel_err(s.particle_pressure_array.cpu().numpy(), o.pressure) < 1e-9
    assert rel_err(s.particle_Cauchy_stress_array.cpu().numpy(), o.sigma) < 1e-9
    assert abs(s.indentation_force[0] - o.force) <= 1e-9 * abs(o.force)


@pytest.mark.parametrize("options", [dict(mobility_law="Uzuoka-Borja"), dict(p2g_projection="lumped"),
                                     dict(mobility_law="Uzuoka-Borja", p2g_projection="lumped")])
def test_terzaghi_driver_options_match_oracle(cuda, options):
    """The J-dependent mobility and the lumped pressure projection of
    problems/consolidation/large_consolidation_cpGIMP_everything_in_one_script.py
    (:330-338 and :292-310), through the 2D u-p solver against the oracle."""
    from geowarp_b200.solvers import quasi_static_coupled_solver_2d
    grid, parts, it, mat, porous, load = cases.terzaghi_dicts(n_cells_y=12)
    porous = dict(porous, **options)
    s = quasi_static_coupled_solver_2d(grid, parts, it, mat, porous, load, cases.terzaghi_boundary_kernel)
    top = cases.top_flags(s.x_particles, grid["end_y"], grid["dx"], parts["PPD"])
    s.particle_pressure_boundary_flag_array[:] = top
    s.particle_traction_flag_array[:] = top
    o = cases.oracle_coupled2d(grid, parts, it, mat, porous, load)
    topn = cases.top_flags(o.x, grid["end_y"], grid["dx"], parts["PPD"])
    o.pbc_flag[:] = topn
    o.trac_flag[:] = topn
    bnd = lambda b: cases.terzaghi_boundary_np(b, grid["n_grid_x"], grid["n_grid_y"])
    for k in range(4):
        s.advance_one_step(k, 600)
        o.advance_one_step(k, 600, set_boundary=bnd)
    assert rel_err(s.particle_pressure_array.cpu().numpy(), o.pressure) < 1e-9
    assert rel_err(s.x_particles.cpu().numpy() - o.x0, o.x - o.x0) < 1e-9
    assert rel_err(s.particle_Cauchy_stress_array.cpu().numpy(), o.sigma) < 1e-9
