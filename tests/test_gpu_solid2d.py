"""GPU parity: 2D solid solver (bar under self-weight, strip footing) against the CPU oracle."""
import numpy as np
import pytest
import torch

import cases
from cases import rel_err

pytestmark = pytest.mark.gpu


def run_gpu_bar(material, steps, n_steps, **kw):
    from geowarp_b200.solvers import quasi_static_solver_2d
    grid, parts, it, mat, load = cases.bar_dicts(material, **kw)
    s = quasi_static_solver_2d(grid, parts, it, mat, load)
    b = np.zeros(s.n_matrix_size, dtype=bool)
    cases.bar_boundary(b, grid["n_grid_x"], grid["n_grid_y"])
    s.dofStruct.boundary_flag_array[:] = torch.as_tensor(b, device=s.x_particles.device)
    for k in range(steps):
        s.advance_one_step(k, n_steps)
    return s


def run_oracle_bar(material, steps, n_steps, **kw):
    grid, parts, it, mat, load = cases.bar_dicts(material, **kw)
    o = cases.oracle_solid2d(grid, parts, it, mat, load)
    cases.bar_boundary(o.boundary, grid["n_grid_x"], grid["n_grid_y"])
    for k in range(steps):
        o.advance_one_step(k, n_steps)
    return o


@pytest.mark.parametrize("material", ["Hencky elasticity", "J2", "Neo-Hookean"])
def test_bar_matches_oracle(cuda, material):
    s = run_gpu_bar(material, 3, 10, height=6.25)
    o = run_oracle_bar(material, 3, 10, height=6.25)
    assert rel_err(s.x_particles.cpu().numpy() - o.x0, o.x - o.x0) < 1e-9
    assert rel_err(s.particle_Cauchy_stress_array.cpu().numpy(), o.sigma) < 1e-9
    assert rel_err(s.deformation_gradient_total_old.cpu().numpy(), o.F_old) < 1e-12
    assert rel_err(s.GIMP_lp.cpu().numpy(), o.lp) < 1e-12


def test_bar_active_set_and_iterations(cuda):
    s = run_gpu_bar("Hencky elasticity", 2, 10, height=6.25)
    o = run_oracle_bar("Hencky elasticity", 2, 10, height=6.25)
    act = s.dofStruct.activate_flag_array.cpu().numpy()
    assert np.array_equal(act, o.active)
    iters = [l for l in s.engine.log]
    assert len(iters) == sum(o.iters)


def test_bar_jacobian_matches_oracle(cuda):
    """Assembled K = -dR/du (field-major, identity rows) against the oracle's
    complex-step element tangents, at the state after one load step."""
    from geowarp_b200.solvers import quasi_static_solver_2d
    grid, parts, it, mat, load = cases.bar_dicts("J2", height=6.25)
    s = run_gpu_bar("J2", 2, 4, height=6.25)
    o = run_oracle_bar("J2", 2, 4, height=6.25)
    # one more P2G + assembly at the same (converged-previous-step) state
    e = s.engine
    s.reset()
    e.sort_and_activate()
    e.build_system()
    e.assemble(s._mat, 2, 4, want_K=True)
    torch.cuda.synchronize()
    rows, cols, vals = (t.cpu().numpy() for t in e.matrix_coo())
    import scipy.sparse as sp
    n = s.n_matrix_size
    Kg = sp.coo_matrix((vals, (rows, cols)), shape=(n, n)).toarray()
    o.u_old[:] = 0.0
    o.u_new[:] = 0.0
    o.p2g()
    R, K, _ = o.assemble(2, 4)
    Ko = K.toarray()
    # the GPU system holds only active nodes; inactive DOFs are identity rows in
    # the reference layout (mpm/mpm_utils.py:1299-1312) and get delta = 0 either way
    act = o.active
    assert np.abs(Kg[np.ix_(act, act)] - Ko[np.ix_(act, act)]).max() <= 1e-9 * np.abs(Ko).max()
    assert np.array_equal(Ko[np.ix_(~act, ~act)], np.eye((~act).sum()))
    assert not Kg[~act].any()
    Rg = s.rhs.cpu().numpy()
    assert np.abs(Rg - R).max() <= 1e-9 * max(np.abs(R).max(), 1e-30)


def test_footing_dp_matches_oracle(cuda):
    from geowarp_b200.solvers import quasi_static_solver_2d
    grid, parts, it, mat, load = cases.footing_dicts(nx=12, ny=6, n_steps=10)
    s = quasi_static_solver_2d(grid, parts, it, mat, load)
    b = np.zeros(s.n_matrix_size, dtype=bool)
    cases.footing_boundary(b, grid)
    s.dofStruct.boundary_flag_array[:] = torch.as_tensor(b, device=s.x_particles.device)
    o = cases.oracle_solid2d(grid, parts, it, mat, load)
    cases.footing_boundary(o.boundary, grid)
    for k in range(3):
        s.advance_one_step(k, 10)
        o.advance_one_step(k, 10)
    assert rel_err(s.x_particles.cpu().numpy() - o.x0, o.x - o.x0) < 1e-9
    assert rel_err(s.particle_Cauchy_stress_array.cpu().numpy(), o.sigma) < 1e-9
    assert abs(s.footing_force - o.force) <= 1e-9 * abs(o.force)


def test_footing_dp_stable_matches_golden(cuda):
    """The benchmark's footing formulation (attractive penalty, footing at the top
    particle layer, Drucker-Prager continued past the tip) on a small block."""
    import os
    from geowarp_b200.solvers import quasi_static_solver_2d
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "footing_dp_stable.npz"))
    grid, parts, it, mat, load = cases.footing_dicts(nx=12, ny=6, n_steps=100, stable=True)
    s = quasi_static_solver_2d(grid, parts, it, mat, load)
    b = np.zeros(s.n_matrix_size, dtype=bool)
    cases.footing_boundary(b, grid)
    s.dofStruct.boundary_flag_array[:] = torch.as_tensor(b, device=s.x_particles.device)
    forces = []
    for k in range(3):
        s.advance_one_step(k, 100)
        forces.append(s.footing_force)
    assert rel_err(s.x_particles.cpu().numpy() - g["x0"], g["x"] - g["x0"]) < 1e-9
    assert rel_err(s.particle_Cauchy_stress_array.cpu().numpy(), g["sigma"]) < 1e-9
    assert np.abs(np.array(forces) - g["force"]).max() <= 1e-9 * np.abs(g["force"]).max()


def test_footing_dp_geostatic_matches_golden(cuda):
    """The benchmark's soil state: self-weight at full magnitude from the first
    load step (gravity_ramp=False) and the K0 geostatic start set by
    problems.geostatic_stress, against the oracle's own restatement."""
    import os
    from geowarp_b200 import problems
    from geowarp_b200.solvers import quasi_static_solver_2d
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "footing_dp_geostatic.npz"))
    grid, parts, it, mat, load = cases.footing_dicts(nx=12, ny=6, n_steps=100, stable=True, geostatic=True)
    s = quasi_static_solver_2d(grid, parts, it, mat, load)
    b = np.zeros(s.n_matrix_size, dtype=bool)
    cases.footing_boundary(b, grid)
    s.dofStruct.boundary_flag_array[:] = torch.as_tensor(b, device=s.x_particles.device)
    problems.geostatic_stress(s, grid["end_y"], parts["p_rho"], load["gravity_mag"],
                              1.0 - np.sin(np.radians(mat["friction_angle"])))
    forces = []
    for k in range(3):
        s.advance_one_step(k, 100)
        forces.append(s.footing_force)
    assert rel_err(s.x_particles.cpu().numpy() - g["x0"], g["x"] - g["x0"]) < 1e-9
    assert rel_err(s.particle_Cauchy_stress_array.cpu().numpy(), g["sigma"]) < 1e-9
    assert np.abs(np.array(forces) - g["force"]).max() <= 1e-9 * np.abs(g["force"]).max()


def test_sort_is_stable_and_deterministic(cuda):
    s = run_gpu_bar("Hencky elasticity", 1, 10, height=6.25)
    e = s.engine
    e.sort_and_activate()
    k1, p1 = e.keys.cpu().numpy().copy(), e.perm.cpu().numpy().copy()
    e.sort_and_activate()
    assert np.array_equal(p1, e.perm.cpu().numpy())
    # reference order: stable argsort of the lower-corner cell key
    x = e.x.cpu().numpy()
    lp = e.lp.cpu().numpy()
    inv = 1.0 / s.dx
    cx = np.clip(np.trunc((x[:, 0] - lp[:, 0]) * inv + 1e-8).astype(np.int64), 0, s.n_grid_x - 1)
    cy = np.clip(np.trunc((x[:, 1] - lp[:, 1]) * inv + 1e-8).astype(np.int64), 0, s.n_grid_y - 1)
    key = cx + cy * s.n_grid_x
    assert np.array_equal(np.argsort(key, kind="stable"), p1)
    assert np.array_equal(key[p1], k1)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_residual_only_assembly_matches_full(cuda, precision):
    """A residual-only deterministic assembly (no tangent) gives the bytes of
    the full assembly's residual, in both precisions.  In mixed precision its
    records use the FP32-tangent layout the workspace is sized for (an earlier
    build wrote FP64-layout records there and overran it)."""
    from geowarp_b200 import batch
    sizes = [(40, 32), (48, 40)]
    bb = batch.BatchedBlocks(sizes, logE=batch.random_fields(sizes, seed=5), precision=precision, device="cuda")
    s = bb.solver
    e = s.engine
    for k in range(2):
        s.advance_one_step(k, 20)
    s._set_step_params()
    s.reset()
    e.sort_and_activate()
    e.build_system()
    n = e.n_rows * e.nf
    e.assemble(s._mat, 2, 20, want_K=True)
    r_full = e._R[:n].clone()
    e.assemble(s._mat, 2, 20, want_K=False)
    torch.cuda.synchronize()
    assert torch.equal(e._R[:n], r_full)
