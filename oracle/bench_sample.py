"""Bounded CPU samples of the benchmark workloads (strip footing,
consolidation column) for the benchmark's CPU-baseline leg (test
infrastructure: the oracle is the checker, timed here only as the reported
CPU baseline).

One Newton iteration of load step 0 of the plane-strain Drucker-Prager strip
footing: residual and complex-step element tangents for every particle
(NumPy, single thread), global assembly and a SciPy sparse direct solve --
the reference's 'scipy' solver path (solvers/quasi_static_solver_2d.py:214-220).
"""
import time

import numpy as np
from scipy.sparse.linalg import spsolve

from . import native
from .mpm import OracleEngine, init_particles_rectangle_2d


def geostatic_b(y, surface_y, rho, gravity, E, nu, K0):
    """Elastic left Cauchy-Green tensors of the geostatic state sigma_yy =
    -rho g (surface_y - y), sigma_xx = sigma_zz = K0 sigma_yy (Hencky law
    inverted with J = 1)."""
    lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    mu = E / (2.0 * (1.0 + nu))
    syy = -rho * gravity * (surface_y - np.asarray(y, dtype=np.float64))
    tau = np.stack([K0 * syy, syy, K0 * syy], axis=-1)
    eps = (tau - lam * tau.sum(-1, keepdims=True) / (3.0 * lam + 2.0 * mu)) / (2.0 * mu)
    b = np.zeros(eps.shape[:-1] + (3, 3))
    for i in range(3):
        b[..., i, i] = np.exp(2.0 * eps[..., i])
    return b


def footing_oracle(n_cells_x=256, n_cells_y=128, dx=0.05, PPD=2, footing_width=1.0, pad=2, gravity=9.81):
    """The strip-footing workload: Drucker-Prager soil (E 2e7 Pa, nu 0.3,
    c 10 kPa, phi 30, psi 0) with self-weight at full magnitude from the first
    load step, starting from the K0 = 1 - sin(phi) geostatic state."""
    n_grid_x, n_grid_y = n_cells_x + 2 * pad, n_cells_y + 2 * pad
    sx, sy = pad * dx, pad * dx
    ex, ey = sx + n_cells_x * dx, sy + n_cells_y * dx
    x = init_particles_rectangle_2d(sx, sy, ex, ey, dx, n_grid_x, n_grid_y, PPD, n_cells_x * n_cells_y * PPD * PPD)
    mat = dict(youngs_modulus=2e7, poisson_ratio=0.3, material_name="Drucker-Prager", friction_angle=30.0,
               dilation_angle=0.0, cohesion=1e4, shape_factor=0.0, tension_cutoff=False)
    xc = 0.5 * (sx + ex)
    load = dict(gravity_mag=gravity, gravity_ramp=False, footing_region_min_x=xc - footing_width / 2,
                footing_region_max_x=xc + footing_width / 2, footing_initial_height=ey - dx / (2 * PPD),
                footing_incr_disp=-0.2 / 100, penalty_factor=1000.0, footing_penalty_stable=True)
    grid = dict(n_grid=(n_grid_x, n_grid_y), h=(dx, dx), h_nodes=(dx, dx), domain_min=(sx, sy), domain_max=(ex, ey))
    o = OracleEngine("solid2d", grid, x, (dx / PPD) ** 2, 2000.0, PPD, mat, load, lp0=dx / PPD / 2.0 - 1e-6,
                     n_iter=20, tol=1e-6)
    nn = (n_grid_x + 1) * (n_grid_y + 1)
    ix = np.tile(np.arange(n_grid_x + 1), n_grid_y + 1)
    iy = np.repeat(np.arange(n_grid_y + 1), n_grid_x + 1)
    dof = ix + iy * (n_grid_x + 1)
    side = (ix <= pad) | (ix >= pad + n_cells_x)
    base = iy <= pad
    o.boundary[dof[side | base]] = True
    o.boundary[dof[base] + nn] = True
    if gravity > 0.0:
        o.b_old = geostatic_b(o.x[:, 1], ey, 2000.0, gravity, 2e7, 0.3, 1.0 - np.sin(np.radians(30.0)))
    return o


def oracle_newton_sample(footing_kwargs=None, full=(256, 128)):
    """Seconds per Newton iteration of the full-size footing, estimated from a
    timed Newton iteration of the 64x32-cell variant (or of the variant given in
    footing_kwargs): the particle-local residual/tangent work scales with the
    particle count, the sparse direct solve with DOFs^1.5 (2D nested dissection)."""
    kw = dict(n_cells_x=64, n_cells_y=32, footing_width=0.25)
    kw.update(footing_kwargs or {})
    o = footing_oracle(**kw)
    o.p2g()
    t0 = time.perf_counter()
    R, K, _ = o.assemble(0, 100)
    t1 = time.perf_counter()
    delta = spsolve(K.tocsc(), R)
    t2 = time.perf_counter()
    o.u_new += delta
    n_full = full[0] * full[1] * 4
    dof_full = 2 * (full[0] + 5) * (full[1] + 5)
    pr = n_full / o.N
    dr = dof_full / o.ndof
    est = (t1 - t0) * pr + (t2 - t1) * dr ** 1.5
    desc = (f"one Newton iteration (residual + complex-step element tangents {t1 - t0:.2f} s, SciPy spsolve "
            f"{t2 - t1:.3f} s) of load step 0 of the {kw['n_cells_x']}x{kw['n_cells_y']}-cell variant "
            f"({o.N} particles, {o.ndof} DOFs), NumPy oracle on 1 host thread; scaled to the 256x128-cell "
            f"workload by x{pr:.0f} (particles) and x{dr ** 1.5:.0f} (solve)")
    return est, desc


def oracle_load_step_sample(footing_kwargs=None, full=(256, 128), step=0, threads=1):
    """Seconds per load step of the full-size footing, from one complete load
    step (P2G, Newton to the tolerance, G2P) of the 64x32-cell variant:
    residual/tangent assembly scaled by the particle count, each sparse direct
    solve by DOFs^1.5.  threads: host threads for the tangent's complex-step
    passes.  Returns (seconds, Newton iterations, description)."""
    import scipy.sparse.linalg as sla
    from . import mpm as M
    kw = dict(n_cells_x=64, n_cells_y=32, footing_width=0.25)
    kw.update(footing_kwargs or {})
    o = footing_oracle(**kw)
    o.threads = threads
    t_solve = [0.0]
    orig = M.spsolve

    def timed_spsolve(A, b):
        t = time.perf_counter()
        x = sla.spsolve(A, b)
        t_solve[0] += time.perf_counter() - t
        return x

    M.spsolve = timed_spsolve
    try:
        t0 = time.perf_counter()
        o.advance_one_step(step, 100)
        total = time.perf_counter() - t0
    finally:
        M.spsolve = orig
    its = o.iters[-1] if getattr(o, "iters", None) else 1
    n_full = full[0] * full[1] * 4
    dof_full = 2 * (full[0] + 5) * (full[1] + 5)
    pr, dr = n_full / o.N, dof_full / o.ndof
    est = (total - t_solve[0]) * pr + t_solve[0] * dr ** 1.5
    desc = (f"one complete load step ({its} Newton iterations; residual + complex-step tangents "
            f"{total - t_solve[0]:.2f} s, SciPy spsolve {t_solve[0]:.3f} s) of load step {step} of the "
            f"{kw['n_cells_x']}x{kw['n_cells_y']}-cell variant ({o.N} particles, {o.ndof} DOFs), NumPy oracle with "
            f"{threads} host thread(s) for the tangent passes (SciPy's direct solve on one); scaled to the 256x128-cell "
            f"workload by x{pr:.0f} (particles) and x{dr ** 1.5:.0f} (solve)")
    return est, its, desc


def consolidation_oracle(grid, parts, it, mat, porous, load):
    """The consolidation column in the oracle, from the solver-constructor
    dictionaries (problems/consolidation/terzaghi_cpGIMP.py:10-73 layout):
    drained, loaded top particles; the caller passes the boundary callback of
    terzaghi_cpGIMP.py:104-119 to advance_one_step."""
    dx = grid["dx"]
    x = init_particles_rectangle_2d(grid["start_x"], grid["start_y"], grid["end_x"], grid["end_y"], dx,
                                    grid["n_grid_x"], grid["n_grid_y"], parts["PPD"], parts["n_particles"])
    og = dict(n_grid=(grid["n_grid_x"], grid["n_grid_y"]), h=(dx, dx), h_nodes=(dx, grid["dy"]),
              domain_min=(grid["domain_min_x"], grid["domain_min_y"]),
              domain_max=(grid["domain_max_x"], grid["domain_max_y"]))
    o = OracleEngine("coupled2d", og, x, parts["p_vol"], parts["p_rho"], parts["PPD"], mat, load,
                     lp0=dx / parts["PPD"] / 2.0 - 1e-6, n_iter=it["n_iter"], tol=it["tol"], dt=it["dt"],
                     phi_initial=porous["phi_initial"], mobility=porous["mobility_constant"])
    top = o.x[:, 1] > grid["end_y"] - dx / parts["PPD"]
    o.pbc_flag[:] = top
    o.trac_flag[:] = top
    return o


def consolidation_boundary_np(boundary, n_grid_x, n_grid_y):
    """x fixed on the side-wall node columns, y fixed on the base row."""
    nn = (n_grid_x + 1) * (n_grid_y + 1)
    ix = np.tile(np.arange(n_grid_x + 1), n_grid_y + 1)
    iy = np.repeat(np.arange(n_grid_y + 1), n_grid_x + 1)
    dof = ix + iy * (n_grid_x + 1)
    boundary[dof[(ix <= 1) | (ix >= 2)]] = True
    boundary[dof[iy <= 0] + nn] = True


def oracle_consolidation_sample(dicts, dts, max_steps=20, budget_s=15.0, threads=1):
    """Seconds per load step of the full consolidation column in the oracle:
    consecutive load steps from the start of the schedule (P2G, Newton to the
    tolerance with a SciPy sparse direct solve, G2P) until max_steps or
    budget_s.  Returns (seconds per step, steps run, description)."""
    grid, parts, it, mat, porous, load = dicts
    o = consolidation_oracle(grid, parts, it, mat, porous, load)
    o.threads = threads
    bnd = lambda b: consolidation_boundary_np(b, grid["n_grid_x"], grid["n_grid_y"])
    t0 = time.perf_counter()
    n = 0
    while n < min(max_steps, len(dts)) and time.perf_counter() - t0 < budget_s:
        o.dt = float(dts[n])
        o.advance_one_step(n, len(dts), set_boundary=bnd)
        n += 1
    sec = (time.perf_counter() - t0) / n
    desc = (f"load steps 0..{n - 1} of the full column ({o.N} particles, {o.ndof} DOFs; "
            f"{sum(o.iters) / n:.1f} Newton iterations per step, complex-step tangents and SciPy spsolve), "
            f"NumPy oracle with {threads} host thread(s) for the tangent passes")
    return sec, n, desc


def bar_oracle(width_cells=4, height_cells=40, dx=0.25, PPD=2, E=1e6, nu=0.3, rho=80.0, gravity=9.81,
               material="Neo-Hookean", n_iter=20, tol=1e-6):
    """The self-weight bar (problems/bar_compaction/bar_compaction_cpGIMP.py
    layout in SI units): rollers on both side walls, fixed base, two empty
    cells around the bar, gravity ramped over the load steps."""
    pad = 2
    n_grid_x, n_grid_y = width_cells + 2 * pad, height_cells + 2 * pad
    sx, sy = pad * dx, pad * dx
    ex, ey = sx + width_cells * dx, sy + height_cells * dx
    x = init_particles_rectangle_2d(sx, sy, ex, ey, dx, n_grid_x, n_grid_y, PPD, width_cells * height_cells * PPD * PPD)
    mat = dict(youngs_modulus=E, poisson_ratio=nu, material_name=material)
    load = dict(gravity_mag=gravity, traction_value_x=0.0, traction_value_y=0.0, point_load_value_x=0.0,
                point_load_value_y=0.0)
    grid = dict(n_grid=(n_grid_x, n_grid_y), h=(dx, dx), h_nodes=(dx, dx), domain_min=(sx, sy), domain_max=(ex, ey))
    o = OracleEngine("solid2d", grid, x, (dx / PPD) ** 2, rho, PPD, mat, load, lp0=dx / PPD / 2.0 - 1e-6,
                     n_iter=n_iter, tol=tol)
    nn = (n_grid_x + 1) * (n_grid_y + 1)
    ix = np.tile(np.arange(n_grid_x + 1), n_grid_y + 1)
    iy = np.repeat(np.arange(n_grid_y + 1), n_grid_x + 1)
    o.boundary[((ix <= pad) | (ix >= pad + width_cells)).nonzero()[0]] = True
    o.boundary[(iy <= pad).nonzero()[0]] = True
    o.boundary[(iy <= pad).nonzero()[0] + nn] = True
    return o


def oracle_bar_sample(n_steps=50, max_steps=50, budget_s=15.0, threads=1):
    """Seconds per load step of the self-weight bar in the oracle:
    consecutive load steps from the start (P2G, Newton with a SciPy sparse
    direct solve, G2P) until max_steps or budget_s.  Returns (seconds per
    step, steps run, description)."""
    o = bar_oracle()
    o.threads = threads
    t0 = time.perf_counter()
    n = 0
    while n < min(max_steps, n_steps) and time.perf_counter() - t0 < budget_s:
        o.advance_one_step(n, n_steps)
        n += 1
    sec = (time.perf_counter() - t0) / n
    desc = (f"load steps 0..{n - 1} of the bar ({o.N} particles, {o.ndof} DOFs; {sum(o.iters) / n:.1f} Newton "
            f"iterations per step, complex-step tangents and SciPy spsolve), NumPy oracle with {threads} host "
            f"thread(s) for the tangent passes")
    return sec, n, desc


def batch_block_oracle(nx, ny, logE, dx=0.05, PPD=2, rho=2000.0, gravity=9.81, nu=0.3, n_iter=20, tol=1e-6):
    """One block of the batched inverse analysis on its own grid (two empty
    cells around it): Hencky elastic with the block's per-particle Young's
    modulus exp(logE), self-weight ramped over the load steps, rollers on its
    side node columns and a fixed base row (the boundary of every packed block)."""
    pad = 2
    n_grid_x, n_grid_y = nx + 2 * pad, ny + 2 * pad
    sx, sy = pad * dx, pad * dx
    ex, ey = sx + nx * dx, sy + ny * dx
    x = init_particles_rectangle_2d(sx, sy, ex, ey, dx, n_grid_x, n_grid_y, PPD, nx * ny * PPD * PPD)
    mat = dict(youngs_modulus=1e7, poisson_ratio=nu, material_name="Hencky elasticity")
    load = dict(gravity_mag=gravity, traction_value_x=0.0, traction_value_y=0.0, point_load_value_x=0.0,
                point_load_value_y=0.0)
    grid = dict(n_grid=(n_grid_x, n_grid_y), h=(dx, dx), h_nodes=(dx, dx), domain_min=(sx, sy), domain_max=(ex, ey))
    o = OracleEngine("solid2d", grid, x, (dx / PPD) ** 2, rho, PPD, mat, load, lp0=dx / PPD / 2.0 - 1e-6,
                     n_iter=n_iter, tol=tol, E_field=np.exp(np.asarray(logE, dtype=np.float64)))
    nn = (n_grid_x + 1) * (n_grid_y + 1)
    ix = np.tile(np.arange(n_grid_x + 1), n_grid_y + 1)
    iy = np.repeat(np.arange(n_grid_y + 1), n_grid_x + 1)
    col = ((ix == pad) | (ix == pad + nx)) & (iy >= pad) & (iy <= pad + ny)
    base = (iy == pad) & (ix >= pad) & (ix <= pad + nx)
    o.boundary[(col | base).nonzero()[0]] = True
    o.boundary[base.nonzero()[0] + nn] = True
    return o


def oracle_batch_sample(sizes, logE, n_steps, budget_s=20.0, threads=1, max_blocks=None, compiled=True):
    """Block load steps per second of the batched inverse analysis in the
    oracle: load step 0 (P2G, Newton to the tolerance with complex-step
    tangents and a SciPy sparse direct solve, G2P) of whole blocks, taken in
    the batch's order until budget_s is spent (at least one block).  The
    blocks are independent, so blocks / seconds is the workload's own unit.
    With compiled (and the library of oracle/native.py built), the
    per-particle residuals and tangents run compiled, in threads over
    particles; otherwise in NumPy, threads over the tangent's passes.
    Returns (block load steps per second, blocks run, description)."""
    offs = np.cumsum([0] + [a * b * 4 for a, b in sizes])
    t0 = time.perf_counter()
    n = 0
    its = []
    parts = 0
    while n < len(sizes) and (max_blocks is None or n < max_blocks):
        nx, ny = sizes[n]
        o = batch_block_oracle(nx, ny, logE[offs[n]:offs[n + 1]])
        o.threads = threads
        o.use_native = compiled
        used = o.use_native and native.supports(o)
        o.advance_one_step(0, n_steps)
        its.append(o.iters[-1] if o.iters else 0)
        parts += o.N
        n += 1
        if time.perf_counter() - t0 > budget_s:
            break
    sec = time.perf_counter() - t0
    desc = (f"load step 0 of {n_steps} (forward: P2G, {np.mean(its):.1f} Newton iterations with complex-step "
            f"tangents and SciPy spsolve, G2P) of blocks 0..{n - 1} of the batch ({parts} particles, sizes "
            f"{', '.join(f'{a}x{b}' for a, b in sizes[:n])}), "
            + (f"oracle with compiled per-particle residuals and tangents (C++, {threads} OpenMP thread(s) over "
               f"particles)" if used else f"NumPy oracle with {threads} host thread(s) for the tangent passes")
            + "; the CPU path has no adjoint")
    return n / sec, n, desc
