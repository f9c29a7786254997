"""Geometric-multigrid flexible GMRES (gw_bsr_gmres_mg_solve) against the
node-block-Jacobi GMRES (gw_bsr_gmres_solve) on the same assembled Newton
systems, and the iteration count it saves."""
import ctypes as C

import numpy as np
import pytest
import torch

import cases
from cases import rel_err

pytestmark = pytest.mark.gpu


def _system_bar(precision):
    from geowarp_b200.solvers import quasi_static_solver_2d
    grid, parts, it, mat, load = cases.bar_dicts("J2", height=12.5)
    s = quasi_static_solver_2d(grid, parts, it, mat, load, precision=precision)
    b = np.zeros(s.n_matrix_size, dtype=bool)
    cases.bar_boundary(b, grid["n_grid_x"], grid["n_grid_y"])
    s.dofStruct.boundary_flag_array[:] = torch.as_tensor(b, device=s.x_particles.device)
    for k in range(3):
        s.advance_one_step(k, 10)
    return s, (3, 10)


def _system_footing(precision):
    from geowarp_b200 import problems
    s = problems.strip_footing_2d(precision=precision, n_cells_x=64, n_cells_y=32, footing_width=0.25)
    for k in range(3):
        s.advance_one_step(k, 100)
    return s, (3, 100)


def _assembled(s, step):
    e = s.engine
    s._set_step_params()
    s.reset()
    e.sort_and_activate()
    e.build_system()
    e.assemble(s._mat, step[0], step[1], want_K=True)
    return e


def _solve(e, precond, rtol):
    n = e.n_rows * e.nf
    x = torch.zeros(n, dtype=torch.float64, device=e.device)
    saved = (e.precond, e.restart)
    e.precond, e.restart = (("mg", 30) if precond == "mg" else (1, 100))
    try:
        it, rr, rc = e.gmres_solve(e.bsr_struct(), e._R, x, rtol)
    finally:
        e.precond, e.restart = saved
    torch.cuda.synchronize()
    return x, it, rr, rc


def _true_relres(e, x):
    from geowarp_b200 import _lib as L
    from geowarp_b200.engine import _p
    n = e.n_rows * e.nf
    y = torch.zeros(n, dtype=torch.float64, device=e.device)
    L.call("gw_bsr_spmv", C.byref(e.bsr_struct()), e.prec, _p(x), _p(y), e.stream)
    b = e._R[:n]
    return float((y - b).norm() / b.norm())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_mg_gmres_matches_jacobi_gmres_on_bar(cuda, precision):
    s, step = _system_bar(precision)
    e = _assembled(s, step)
    from geowarp_b200 import _lib as L
    x_j, it_j, rr_j, rc_j = _solve(e, "block", 1e-12)
    x_m, it_m, rr_m, rc_m = _solve(e, "mg", 1e-12)
    # second Gram-Schmidt passes are taken only where the projection cancelled
    assert 0 <= L.load().gw_gmres_last_reorths() <= it_m
    assert rc_j == 0 and rc_m == 0
    assert _true_relres(e, x_m) < 1e-10
    assert rel_err(x_m.cpu().numpy(), x_j.cpu().numpy()) < 1e-9
    assert it_m < it_j


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_mg_gmres_on_footing_converges_in_few_iterations(cuda, precision):
    """The Drucker-Prager footing Jacobian (penalty footing, plastic zone) is
    ill-conditioned; the V-cycle cuts the Krylov count by an order of magnitude
    and both solutions satisfy the system to the requested tolerance."""
    s, step = _system_footing(precision)
    e = _assembled(s, step)
    rtol = 1e-10
    x_j, it_j, rr_j, rc_j = _solve(e, "block", rtol)
    x_m, it_m, rr_m, rc_m = _solve(e, "mg", rtol)
    assert rc_j == 0 and rc_m == 0
    assert _true_relres(e, x_m) < 10 * rtol
    assert _true_relres(e, x_j) < 10 * rtol
    assert 5 * it_m < it_j


def test_mg_default_solver_reproduces_block_jacobi_terzaghi(cuda):
    """Whole-solver check on the coupled u-p column: the Newton solution with
    the default multigrid preconditioner equals the block-Jacobi one."""
    from geowarp_b200.solvers import quasi_static_coupled_solver_2d
    out = {}
    for precond in ("mg", "block"):
        grid, parts, it, mat, porous, load = cases.terzaghi_dicts(n_cells_y=12)
        s = quasi_static_coupled_solver_2d(grid, parts, it, mat, porous, load, cases.terzaghi_boundary_kernel,
                                           precond=precond)
        top = cases.top_flags(s.x_particles, grid["end_y"], grid["dx"], parts["PPD"])
        s.particle_pressure_boundary_flag_array[:] = top
        s.particle_traction_flag_array[:] = top
        for k in range(4):
            s.advance_one_step(k, 600)
        out[precond] = (s.particle_pressure_array.cpu().numpy(), (s.x_particles - s.x0).cpu().numpy())
    assert rel_err(out["mg"][0], out["block"][0]) < 1e-9
    assert rel_err(out["mg"][1], out["block"][1]) < 1e-9


def test_mg_plan_reuse_and_rejection(cuda):
    """A plan built once serves repeated solves on the same pattern; a plan from
    another workspace is refused before any launch."""
    from geowarp_b200 import _lib as L
    from geowarp_b200.engine import _p
    s, step = _system_footing("fp64")
    e = _assembled(s, step)
    lib = L.load()
    g = e.grid_struct()
    A = e.bsr_struct()
    nbytes = lib.gw_gmres_mg_workspace_bytes(C.byref(g), e.n_rows, e.nf, 30)
    ws = torch.zeros(nbytes, dtype=torch.uint8, device=e.device)
    plan = L.MgPlan()
    L.call("gw_mg_plan_build", C.byref(g), C.byref(A), _p(ws), nbytes, C.byref(plan), e.stream)
    assert plan.levels >= 2 and plan.dense_n <= 160 and plan.fine_n_rows == e.n_rows
    n = e.n_rows * e.nf
    xs = []
    for _ in range(2):
        x = torch.zeros(n, dtype=torch.float64, device=e.device)
        it, rr = C.c_int32(0), C.c_double(0.0)
        rc = lib.gw_bsr_gmres_mg_solve(C.byref(g), C.byref(A), e.prec, C.byref(plan), _p(e._R), _p(x), 1e-10, 500,
                                       30, _p(ws), nbytes, C.byref(it), C.byref(rr), e.stream)
        assert rc == 0
        xs.append(x.cpu().numpy())
    assert np.array_equal(xs[0], xs[1])
    assert plan.last_iters > 0  # the solve leaves its iteration count in the plan
    # a matrix with other pattern arrays (a copy of the column array) is refused
    cols2 = e._cols.clone()
    A2 = e.bsr_struct()
    A2.cols = _p(cols2)
    x = torch.zeros(n, dtype=torch.float64, device=e.device)
    rc = lib.gw_bsr_gmres_mg_solve(C.byref(g), C.byref(A2), e.prec, C.byref(plan), _p(e._R), _p(x), 1e-10, 500,
                                   30, _p(ws), nbytes, C.byref(it), C.byref(rr), e.stream)
    assert rc == L.GW_EINVAL
    ws2 = torch.zeros(nbytes, dtype=torch.uint8, device=e.device)
    x = torch.zeros(n, dtype=torch.float64, device=e.device)
    it, rr = C.c_int32(0), C.c_double(0.0)
    rc = lib.gw_bsr_gmres_mg_solve(C.byref(g), C.byref(A), e.prec, C.byref(plan), _p(e._R), _p(x), 1e-12, 200, 30,
                                   _p(ws2), nbytes, C.byref(it), C.byref(rr), e.stream)
    assert rc == L.GW_EINVAL
    assert b"plan" in lib.gw_status_string(rc)


def test_mg_workspace_too_small_is_rejected(cuda):
    from geowarp_b200 import _lib as L
    from geowarp_b200.engine import _p
    s, step = _system_bar("fp64")
    e = _assembled(s, step)
    lib = L.load()
    g = e.grid_struct()
    need = lib.gw_gmres_mg_workspace_bytes(C.byref(g), e.n_rows, e.nf, 30)
    assert need > 0
    ws = torch.zeros(need // 2, dtype=torch.uint8, device=e.device)
    n = e.n_rows * e.nf
    x = torch.zeros(n, dtype=torch.float64, device=e.device)
    it, rr = C.c_int32(0), C.c_double(0.0)
    rc = lib.gw_bsr_gmres_mg_solve(C.byref(g), C.byref(e.bsr_struct()), e.prec, None, _p(e._R), _p(x), 1e-10, 100,
                                   30, _p(ws), ws.numel(), C.byref(it), C.byref(rr), e.stream)
    assert rc == L.GW_EINVAL
    assert b"workspace" in lib.gw_status_string(rc)


def test_launch_knobs_change_speed_not_results(cuda):
    """The autotuner's knobs (CTA sizes, the dense coarsest level bound) leave
    the converged load steps as they are: same forward state and gradient as
    with the default knobs, to the Krylov tolerance."""
    from geowarp_b200 import _lib as L
    from geowarp_b200 import problems
    from geowarp_b200.adjoint import LoadStepAdjoint
    lib = L.load()
    defaults = {k: lib.gw_tune_get(k) for k in range(L.TUNE_COUNT)}

    def run():
        s = problems.bar_compaction_2d(precision="fp64", device=cuda)
        adj = LoadStepAdjoint(s)
        for k in range(3):
            adj.forward_step(k, 50, keep=False)
            adj.seed_displacement_misfit()
            adj.backward_step()
        return (s.x_particles - s.x0).cpu().numpy(), adj.grad_E.cpu().numpy()

    try:
        u0, g0 = run()
        for k, v in [(L.TUNE_PARTICLE_BLOCK, 64), (L.TUNE_ADJOINT_BLOCK, 64), (L.TUNE_ROW_WARPS, 2),
                     (L.TUNE_MG_COARSE, 40)]:
            assert lib.gw_tune_set(k, v) == L.GW_OK
        u1, g1 = run()
    finally:
        for k, v in defaults.items():
            lib.gw_tune_set(k, v)
    assert rel_err(u1, u0) < 1e-9
    assert rel_err(g1, g0) < 1e-7


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fused_coarse_tail_is_bitwise_the_per_phase_vcycle(cuda, precision):
    """The coarse levels run as one cluster launch (GW_TUNE_MG_TAIL) give the
    same bytes as one launch per phase, in fewer launches."""
    from geowarp_b200 import _lib as L
    lib = L.load()
    default = lib.gw_tune_get(L.TUNE_MG_TAIL)
    s, step = _system_footing(precision)
    e = _assembled(s, step)
    out = {}
    try:
        for tail in (0, 4096):
            assert lib.gw_tune_set(L.TUNE_MG_TAIL, tail) == L.GW_OK
            n0 = lib.gw_launch_count()
            x, it, rr, rc = _solve(e, "mg", 1e-10)
            out[tail] = (x.cpu().numpy(), it, rc, lib.gw_launch_count() - n0)
    finally:
        lib.gw_tune_set(L.TUNE_MG_TAIL, default)
    (x0, it0, rc0, n_sep), (x1, it1, rc1, n_tail) = out[0], out[4096]
    assert rc0 == 0 and rc1 == 0 and it0 == it1
    assert np.array_equal(x0, x1)
    assert n_tail < n_sep


def test_mixed_options_change_iterates_not_the_converged_state(cuda):
    """The mixed-precision engine's chord final update and the V-cycle's BF16
    fine-level copy change how each load step is solved, not what it
    converges to: with both on and both off, the bar's displacement and stress
    after a few load steps agree far below the Newton tolerance's effect."""
    from geowarp_b200 import _lib as L
    from geowarp_b200 import problems
    lib = L.load()
    default = lib.gw_tune_get(L.TUNE_MG_BF16)
    out = {}
    try:
        for on in (False, True):
            assert lib.gw_tune_set(L.TUNE_MG_BF16, int(on)) == L.GW_OK
            s = problems.bar_compaction_2d(precision="mixed", device=cuda, tol=1e-8)
            s.engine.final_chord = on
            for k in range(4):
                s.advance_one_step(k, 20)
            out[on] = ((s.x_particles - s.x0).cpu().numpy(), s.particle_Cauchy_stress_array.cpu().numpy())
    finally:
        lib.gw_tune_set(L.TUNE_MG_BF16, default)
    assert rel_err(out[True][0], out[False][0]) < 1e-8
    assert rel_err(out[True][1], out[False][1]) < 1e-8
