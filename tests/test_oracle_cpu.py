"""CPU checks of the oracle: analytic known answers from the reference's own
driver scripts, exactness of its complex-step tangents, and the committed
golden fixtures."""
import os

import numpy as np
import pytest

import cases
from oracle.eig import eigh3

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


@pytest.mark.parametrize("material", ["Hencky elasticity", "J2"])
def test_bar_self_weight_known_answer(material):
    """Relative L1 error of sigma_yy against rho g (H - (y0 - start_y)), the
    check of problems/bar_compaction_J2/bar_compaction_cpGIMP_J2.py:113-131."""
    H = 12.5
    grid, parts, it, mat, load = cases.bar_dicts(material, height=H)
    o = cases.oracle_solid2d(grid, parts, it, mat, load)
    cases.bar_boundary(o.boundary, grid["n_grid_x"], grid["n_grid_y"])
    n_steps = 10
    for k in range(n_steps):
        o.advance_one_step(k, n_steps)
    rho, g = parts["p_rho"], load["gravity_mag"]
    ana = rho * (-g) * (H - (o.x0[:, 1] - grid["start_y"]))
    err = np.abs(o.sigma[:, 1, 1] - ana).sum() / (g * rho * H * o.N)
    assert err < 5e-3, err
    assert max(o.iters) <= 6  # quadratic Newton convergence with the exact tangent


def test_oracle_reproduces_golden_bar():
    g = golden("bar_hencky")
    grid, parts, it, mat, load = cases.bar_dicts("Hencky elasticity", height=12.5)
    o = cases.oracle_solid2d(grid, parts, it, mat, load)
    cases.bar_boundary(o.boundary, grid["n_grid_x"], grid["n_grid_y"])
    steps, n_steps = g["steps"]
    for k in range(steps):
        o.advance_one_step(k, n_steps)
    assert np.array_equal(o.active, g["active"])
    assert np.abs(o.x - g["x"]).max() < 1e-13
    assert np.abs(o.sigma - g["sigma"]).max() < 1e-11 * np.abs(g["sigma"]).max()


def test_oracle_reproduces_golden_terzaghi():
    g = golden("terzaghi")
    grid, parts, it, mat, porous, load = cases.terzaghi_dicts(n_cells_y=12)
    o = cases.oracle_coupled2d(grid, parts, it, mat, porous, load)
    top = cases.top_flags(o.x, grid["end_y"], grid["dx"], parts["PPD"])
    o.pbc_flag[:] = top
    o.trac_flag[:] = top
    for k in range(4):
        o.advance_one_step(k, 600, set_boundary=lambda b: cases.terzaghi_boundary_np(b, grid["n_grid_x"], grid["n_grid_y"]))
    assert np.array_equal(o.boundary, g["boundary"])
    assert np.abs(o.pressure - g["pressure"]).max() < 1e-11 * np.abs(g["pressure"]).max()


def _fd_check(o, step, n_steps, rng, h=1e-7):
    R, K, _ = o.assemble(step, n_steps)
    free = o.active & ~o.boundary
    v = np.where(free, rng.normal(size=o.ndof), 0.0)
    u0 = o.u_new.copy()
    o.u_new = u0 + h * v
    Rp, _, _ = o.assemble(step, n_steps, want_K=False)
    o.u_new = u0 - h * v
    Rm, _, _ = o.assemble(step, n_steps, want_K=False)
    o.u_new = u0
    fd = -(Rp - Rm) / (2 * h)
    Kv = K @ v
    return np.abs(Kv[free] - fd[free]).max() / np.abs(fd[free]).max()


def test_oracle_tangent_matches_fd_solid():
    rng = np.random.default_rng(0)
    grid, parts, it, mat, load = cases.bar_dicts("J2", height=6.25)
    o = cases.oracle_solid2d(grid, parts, it, mat, load)
    cases.bar_boundary(o.boundary, grid["n_grid_x"], grid["n_grid_y"])
    o.advance_one_step(0, 4)
    o.u_new[:] = 0.0
    o.p2g()
    assert _fd_check(o, 1, 4, rng) < 1e-6


def test_oracle_tangent_matches_fd_footing():
    rng = np.random.default_rng(1)
    grid, parts, it, mat, load = cases.footing_dicts(nx=8, ny=4, n_steps=10)
    o = cases.oracle_solid2d(grid, parts, it, mat, load)
    cases.footing_boundary(o.boundary, grid)
    o.p2g()
    o.u_new = rng.normal(scale=1e-4, size=o.ndof) * (o.active & ~o.boundary)
    assert _fd_check(o, 0, 10, rng, h=1e-9) < 1e-5


def test_oracle_tangent_matches_fd_coupled():
    rng = np.random.default_rng(2)
    grid, parts, it, mat, porous, load = cases.terzaghi_dicts(n_cells_y=6)
    o = cases.oracle_coupled2d(grid, parts, it, mat, porous, load)
    top = cases.top_flags(o.x, grid["end_y"], grid["dx"], parts["PPD"])
    o.pbc_flag[:] = top
    o.trac_flag[:] = top
    cases.terzaghi_boundary_np(o.boundary, grid["n_grid_x"], grid["n_grid_y"])
    o.p2g()
    o.u_new = o.u_new + rng.normal(scale=1e-3, size=o.ndof) * (o.active & ~o.boundary)
    assert _fd_check(o, 0, 600, rng, h=1e-8) < 1e-5


def test_eigh3_reconstruction_and_complex_step():
    rng = np.random.default_rng(3)
    A = rng.normal(size=(64, 3, 3))
    A = A + A.transpose(0, 2, 1)
    lam, V = eigh3(A)
    assert np.abs(np.einsum("nia,na,nja->nij", V, lam, V) - A).max() < 1e-13
    E = rng.normal(size=(64, 3, 3))
    E = E + E.transpose(0, 2, 1)
    lc, Vc = eigh3(A + 1e-30j * E)
    dl = np.imag(lc) / 1e-30
    ana = np.einsum("nia,nij,nja->na", V, E, V)  # dlambda_a = v_a^T E v_a
    assert np.abs(dl - ana).max() < 1e-12


def test_triaxial_dp_reaches_the_cone():
    g = golden("triaxial_dp")
    phi = np.deg2rad(35.0)
    M = 6 * np.sin(phi) / (3 - np.sin(phi))
    assert abs(g["Q"][-1] / g["P"][-1] - M) < 2e-3 * M
    assert np.all(np.diff(g["Q"][:4]) > 0)


def test_geostatic_state_inverts_hencky_and_is_in_equilibrium():
    """The K0 geostatic start of the footing workload: the product's and the
    oracle's left Cauchy-Green tensors agree, reproduce sigma_yy = -rho g depth
    and K0 sigma_yy through the Hencky law, and give a small initial residual
    compared with the self-weight (cpGIMP integrates the linear stress field
    of the layer exactly, so the discrete state is in equilibrium)."""
    import torch
    from geowarp_b200.problems import geostatic_left_cauchy_green
    from oracle.bench_sample import geostatic_b
    E, nu, K0, rho, g = 2e7, 0.3, 0.5, 2000.0, 9.81
    y = np.linspace(0.1, 1.2, 23)
    b_o = geostatic_b(y, 1.3, rho, g, E, nu, K0)
    b_p = geostatic_left_cauchy_green(torch.as_tensor(y), 1.3, rho, g, E, nu, K0).numpy()
    assert np.abs(b_o - b_p).max() < 1e-15
    lam, mu = E * nu / ((1 + nu) * (1 - 2 * nu)), E / (2 * (1 + nu))
    eps = 0.5 * np.log(np.diagonal(b_o, axis1=1, axis2=2))
    tau = lam * eps.sum(-1, keepdims=True) + 2 * mu * eps
    syy = -rho * g * (1.3 - y)
    assert np.abs(tau[:, 1] - syy).max() < 1e-9 * rho * g
    assert np.abs(tau[:, 0] - K0 * syy).max() < 1e-9 * rho * g
    # equilibrium of the small geostatic footing block before the footing moves
    grid, parts, it, mat, load = cases.footing_dicts(nx=12, ny=6, n_steps=100, stable=True, geostatic=True)
    load = dict(load, footing_incr_disp=0.0)
    o = cases.oracle_solid2d(grid, parts, it, mat, load)
    cases.footing_boundary(o.boundary, grid)
    o.b_old = geostatic_b(o.x[:, 1], grid["end_y"], rho, g, E, nu, K0)
    o.p2g()
    R, _, _ = o.assemble(0, 100, want_K=False)
    weight = rho * g * parts["p_vol"] * parts["n_particles"]
    assert np.linalg.norm(R) < 1e-9 * weight


def test_threaded_tangent_passes_give_the_same_jacobian():
    """The oracle's complex-step passes on several host threads (the timing
    runs) assemble exactly the residual and Jacobian of the serial passes."""
    from oracle.bench_sample import footing_oracle
    o = footing_oracle(n_cells_x=16, n_cells_y=8, footing_width=0.25)
    o.p2g()
    R1, K1, _ = o.assemble(0, 100)
    o.threads = 4
    R2, K2, _ = o.assemble(0, 100)
    assert np.array_equal(R1, R2)
    assert (K1 != K2).nnz == 0 and K1.nnz == K2.nnz


def test_compiled_per_particle_path_matches_the_numpy_oracle():
    """oracle/solid2d_cpu.cpp (the CPU baseline's per-particle residuals and
    complex-step tangents) against the NumPy oracle: one assembly from a
    perturbed state agrees to round-off, and whole load steps of a batch
    block follow the same Newton iterations to the same state."""
    from oracle import native
    from oracle.bench_sample import batch_block_oracle
    native.build()
    assert native.load() is not None
    rng = np.random.default_rng(3)
    logE = np.log(1e7) + 0.3 * rng.normal(size=14 * 10 * 4)

    o = batch_block_oracle(14, 10, logE)
    o.advance_one_step(0, 20)  # F, b and x away from the initial state
    o.u_old[:] = 0.0
    o.u_new[:] = 0.0
    o.p2g()
    free = o.active & ~o.boundary
    o.u_new[free] = 1e-4 * rng.normal(size=int(free.sum()))
    assert native.supports(o)
    R0, K0, a0 = o.assemble(1, 20)
    o.use_native, o.threads = True, 3
    R1, K1, a1 = o.assemble(1, 20)
    assert np.abs(R1 - R0).max() <= 1e-12 * np.abs(R0).max()
    assert K1.nnz == K0.nnz
    assert abs(K1 - K0).max() <= 1e-12 * abs(K0).max()
    for k in ("F_new", "b_new", "sigma"):
        assert np.abs(a1[k] - np.real(a0[k])).max() <= 1e-12 * np.abs(np.real(a0[k])).max()

    runs = {}
    for use in (False, True):
        o = batch_block_oracle(14, 10, logE)
        o.use_native, o.threads = use, 2
        for k in range(3):
            o.advance_one_step(k, 20)
        runs[use] = (o.x.copy(), o.sigma.copy(), list(o.iters))
    assert runs[True][2] == runs[False][2]
    assert np.abs(runs[True][0] - runs[False][0]).max() <= 1e-12 * np.abs(runs[False][0]).max()
    assert np.abs(runs[True][1] - runs[False][1]).max() <= 1e-9 * np.abs(runs[False][1]).max()
