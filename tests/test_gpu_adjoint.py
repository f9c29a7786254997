"""GPU: the hand-written load-step adjoint against central finite differences
of the full GPU simulation, for a per-particle log-Young's-modulus field."""
import numpy as np
import pytest
import torch

import cases

pytestmark = pytest.mark.gpu


def make_solver(kind, precision="fp64"):
    from geowarp_b200.solvers import quasi_static_solver_2d
    if kind == "footing":
        grid, parts, it, mat, load = cases.footing_dicts(nx=12, ny=6, n_steps=10, tol=1e-9, n_iter=25)
        s = quasi_static_solver_2d(grid, parts, it, mat, load, precision=precision)
        b = np.zeros(s.n_matrix_size, dtype=bool)
        cases.footing_boundary(b, grid)
    else:
        grid, parts, it, mat, load = cases.bar_dicts(kind, height=6.25, tol=1e-11, E=10.0, nu=0.2)
        s = quasi_static_solver_2d(grid, parts, it, mat, load, precision=precision)
        b = np.zeros(s.n_matrix_size, dtype=bool)
        cases.bar_boundary(b, grid["n_grid_x"], grid["n_grid_y"])
    s.dofStruct.boundary_flag_array[:] = torch.as_tensor(b, device=s.x_particles.device)
    s.engine.krylov_rtol = 1e-13
    return s


def reset(s):
    e = s.engine
    e.x.copy_(e.x0)
    ident = torch.tensor([[1.0 + 1e-7, 0, 0], [0, 1.0 - 1e-6, 0], [0, 0, 1.0]], dtype=torch.float64, device=e.device)
    for t in (e.F_old, e.F_new, e.b_old, e.b_new):
        t[:] = ident
    e.lp.fill_(s.GIMP_lp_initial)
    e.sigma.zero_()


@pytest.mark.parametrize("kind,steps,n_steps", [("Hencky elasticity", 3, 6), ("J2", 3, 6), ("footing", 3, 10)])
def test_adjoint_matches_central_fd(cuda, kind, steps, n_steps):
    from geowarp_b200.adjoint import DisplacementMisfit
    s = make_solver(kind)
    rng = np.random.default_rng(5)
    E0 = s.youngs_modulus
    N = s.n_particles
    logE = torch.tensor(np.log(E0) + 0.1 * rng.normal(size=N), device=cuda, requires_grad=True)
    target = torch.tensor(rng.normal(scale=1e-3, size=(N, 2)), device=cuda)
    loss = DisplacementMisfit.apply(logE, s, target, n_steps, steps, reset)
    loss.backward()
    g = logE.grad.detach().clone()
    v = torch.tensor(rng.normal(size=N), device=cuda)
    h = 1e-5
    with torch.no_grad():
        lp = DisplacementMisfit.apply(logE.detach() + h * v, s, target, n_steps, steps, reset)
        lm = DisplacementMisfit.apply(logE.detach() - h * v, s, target, n_steps, steps, reset)
    fd = float((lp - lm) / (2 * h))
    ad = float((g * v).sum())
    assert abs(ad - fd) <= 2e-5 * abs(fd), (ad, fd)


def test_mixed_adjoint_close_to_fp64(cuda):
    from geowarp_b200.adjoint import DisplacementMisfit
    grads = {}
    for prec in ("fp64", "mixed"):
        s = make_solver("footing", precision=prec)
        rng = np.random.default_rng(6)
        N = s.n_particles
        logE = torch.tensor(np.log(s.youngs_modulus) + 0.1 * rng.normal(size=N), device=cuda, requires_grad=True)
        target = torch.zeros((N, 2), dtype=torch.float64, device=cuda)
        DisplacementMisfit.apply(logE, s, target, 10, 2, reset).backward()
        grads[prec] = logE.grad.detach()
    # the mixed adjoint solves K^T lambda = u_bar with the FP32 Jacobian to a
    # relative 1e-6: the gradient agrees to a few 1e-4
    rel = float((grads["mixed"] - grads["fp64"]).abs().max() / grads["fp64"].abs().max())
    assert rel < 5e-3, rel
