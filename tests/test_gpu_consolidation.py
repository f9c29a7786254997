"""The consolidation column (linear elastic skeleton, geometrically growing
time increments) on the multigrid-preconditioned u-p solver: parity with the
oracle on a short column, and on the full 1 x 200-cell column Terzaghi's
analytic pore pressure plus the error of the mixed-precision engine against
the FP64 one."""
import numpy as np
import pytest
import torch

import cases
from cases import rel_err

pytestmark = pytest.mark.gpu

Q = 1e4  # surface load (Pa)


def _oracle(**kw):
    from geowarp_b200 import problems
    grid, parts, it, mat, porous, load, dts, cv, H = problems.consolidation_column_dicts(**kw)
    o = cases.oracle_coupled2d(grid, parts, it, mat, porous, load)
    top = cases.top_flags(o.x, grid["end_y"], grid["dx"], parts["PPD"])
    o.pbc_flag[:] = top
    o.trac_flag[:] = top
    return o, dts, lambda b: cases.terzaghi_boundary_np(b, grid["n_grid_x"], grid["n_grid_y"])


# The reference's stopping rule (absolute ||R|| < 1e-8, with force rows of
# order 1e2 N and mass-balance rows of order 1e-10) leaves this u-p system at
# its FP64 rounding floor: the fields are determined only to the spread that
# further Newton iterations at the floor produce (about 2e-5 relative on the
# 40-cell column).  The test measures that spread with a second oracle run
# (tol 1e-13, six Newton iterations per step) and asserts the GPU within three
# times it, and never looser than 1e-9.


def _fields(x, x0, p, sigma):
    return np.asarray(p), np.asarray(x) - np.asarray(x0), np.asarray(sigma)


def test_short_column_matches_oracle(cuda):
    from geowarp_b200 import problems
    kw = dict(n_cells=40, n_steps=6)
    s, dts, cv, H = problems.consolidation_column_2d(precision="fp64", **kw)
    o, dts_o, bnd = _oracle(**kw)
    o_floor, _, _ = _oracle(tol=1e-13, n_iter=6, **kw)
    assert np.array_equal(dts, dts_o)
    for k in range(len(dts)):
        s.dt = o.dt = o_floor.dt = float(dts[k])
        s.advance_one_step(k, len(dts))
        o.advance_one_step(k, len(dts), set_boundary=bnd)
        o_floor.advance_one_step(k, len(dts), set_boundary=bnd)
    assert np.array_equal(s.dofStruct.boundary_flag_array.cpu().numpy(), o.boundary)
    gpu = _fields(s.x_particles.cpu().numpy(), o.x0, s.particle_pressure_array.cpu().numpy(),
                  s.particle_Cauchy_stress_array.cpu().numpy())
    ref = _fields(o.x, o.x0, o.pressure, o.sigma)
    flo = _fields(o_floor.x, o.x0, o_floor.pressure, o_floor.sigma)
    for name, g, r, f in zip(("pore pressure", "displacement", "stress"), gpu, ref, flo):
        err, spread = rel_err(g, r), rel_err(f, r)
        print(f"short column, {name}: GPU vs oracle {err:.2e}, oracle spread at the FP64 floor {spread:.2e}")
        assert err <= max(3.0 * spread, 1e-9), name


def _run_column(precision):
    from geowarp_b200 import problems
    s, dts, cv, H = problems.consolidation_column_2d(precision=precision)
    s.engine.krylov_max_iter = 400
    t, errs = 0.0, []
    for k in range(len(dts)):
        s.dt = float(dts[k])
        t += dts[k]
        n0 = len(s.engine.log)
        s.advance_one_step(k, len(dts))
        log = s.engine.log[n0:]
        assert log[-1][2] < 1e-8, f"step {k}: Newton did not converge ({log})"
        if k % 10 == 9:
            y = s.x0[:, 1].cpu().numpy()
            pa = problems.terzaghi_pressure(H - y, t, H, cv, Q)
            errs.append((cv * t / H ** 2, np.abs(s.particle_pressure_array.cpu().numpy() - pa).max() / Q))
    return s, errs


def test_full_column_follows_terzaghi_and_mixed_tracks_fp64(cuda):
    s64, errs64 = _run_column("fp64")
    smx, errs_mx = _run_column("mixed")
    # Terzaghi: once the drainage front spans a few cells (T >= 1e-3) the
    # particle pore pressure stays within 1.5% of the surface load
    late = [e for T, e in errs64 if T >= 1e-3]
    assert late and max(late) < 0.015, errs64
    assert max(e for _, e in errs64) < 0.1, errs64
    # mixed precision (FP32 assembly / SpMV, FP64 residual and refinement)
    # against the FP64 engine, within the determinacy of the FP64 fields
    p64 = s64.particle_pressure_array.cpu().numpy()
    pmx = smx.particle_pressure_array.cpu().numpy()
    u64 = (s64.x_particles - s64.x0).cpu().numpy()
    umx = (smx.x_particles - smx.x0).cpu().numpy()
    p_err = np.abs(pmx - p64).max() / Q
    u_err = rel_err(umx, u64)
    print(f"mixed vs fp64: pore pressure {p_err:.2e} of the load, settlement {u_err:.2e}")
    assert p_err < 1e-5
    assert u_err < 1e-4
