"""Generate the golden fixtures of tests/golden/*.npz from the CPU oracle.

The reference (Warp) cannot run here, so the fixtures are oracle outputs on
small seeded problems built with the reference's own setups (bar compaction,
Terzaghi column, 3D indentation, triaxial drivers) plus the documented
extensions (Drucker-Prager strip footing).  Run from the repository root:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import cases  # noqa: E402
from oracle.bench_sample import geostatic_b  # noqa: E402
from oracle.triaxial import triaxial_dp, triaxial_norsand  # noqa: E402


def save(name, **arrays):
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
    print("wrote", name, {k: np.shape(v) for k, v in arrays.items()})


def bar(material, steps=5, n_steps=10):
    grid, parts, it, mat, load = cases.bar_dicts(material, height=12.5)
    o = cases.oracle_solid2d(grid, parts, it, mat, load)
    cases.bar_boundary(o.boundary, grid["n_grid_x"], grid["n_grid_y"])
    for k in range(steps):
        o.advance_one_step(k, n_steps)
    return dict(x=o.x, x0=o.x0, sigma=o.sigma, F=o.F_old, b=o.b_old, lp=o.lp, active=o.active,
                iters=np.array(o.iters), steps=np.array([steps, n_steps]))


def footing(steps=3, n_steps=10, **kw):
    grid, parts, it, mat, load = cases.footing_dicts(nx=12, ny=6, n_steps=n_steps, **kw)
    o = cases.oracle_solid2d(grid, parts, it, mat, load)
    cases.footing_boundary(o.boundary, grid)
    if kw.get("geostatic"):
        o.b_old = geostatic_b(o.x[:, 1], grid["end_y"], parts["p_rho"], load["gravity_mag"], mat["youngs_modulus"],
                              mat["poisson_ratio"], 1.0 - np.sin(np.radians(mat["friction_angle"])))
    forces = []
    for k in range(steps):
        o.advance_one_step(k, n_steps)
        forces.append(o.force)
    return dict(x=o.x, x0=o.x0, sigma=o.sigma, F=o.F_old, lp=o.lp, force=np.array(forces), iters=np.array(o.iters))


def terzaghi(steps=4):
    grid, parts, it, mat, porous, load = cases.terzaghi_dicts(n_cells_y=12)
    o = cases.oracle_coupled2d(grid, parts, it, mat, porous, load)
    top = cases.top_flags(o.x, grid["end_y"], grid["dx"], parts["PPD"])
    o.pbc_flag[:] = top
    o.trac_flag[:] = top
    for k in range(steps):
        o.advance_one_step(k, 600, set_boundary=lambda b: cases.terzaghi_boundary_np(b, grid["n_grid_x"], grid["n_grid_y"]))
    return dict(x=o.x, x0=o.x0, sigma=o.sigma, pressure=o.pressure, boundary=o.boundary, active=o.active,
                iters=np.array(o.iters))


def indentation(steps=2):
    grid, parts, it, mat, porous, load = cases.indentation_dicts(n=4)
    o = cases.oracle_coupled3d(grid, parts, it, mat, porous, load)
    o.pbc_flag[:] = o.x[:, 2] > grid["end_z"] - grid["dz"] / parts["PPD"]
    forces = []
    for k in range(steps):
        o.advance_one_step(k, 25, set_boundary=lambda b: cases.indentation_boundary_np(b, grid))
        forces.append(o.force)
    return dict(x=o.x, x0=o.x0, sigma=o.sigma, pressure=o.pressure, force=np.array(forces), active=o.active,
                iters=np.array(o.iters))


def jacobian_bar_j2():
    grid, parts, it, mat, load = cases.bar_dicts("J2", height=6.25)
    o = cases.oracle_solid2d(grid, parts, it, mat, load)
    cases.bar_boundary(o.boundary, grid["n_grid_x"], grid["n_grid_y"])
    for k in range(2):
        o.advance_one_step(k, 4)
    o.u_old[:] = 0.0
    o.u_new[:] = 0.0
    o.p2g()
    R, K, _ = o.assemble(2, 4)
    K = K.tocoo()
    return dict(R=R, rows=K.row, cols=K.col, vals=K.data, n=np.array([K.shape[0]]))


if __name__ == "__main__":
    save("bar_hencky", **bar("Hencky elasticity"))
    save("bar_j2", **bar("J2"))
    save("bar_neohookean", **bar("Neo-Hookean"))
    save("footing_dp", **footing())
    save("footing_dp_stable", **footing(stable=True, n_steps=100))
    save("footing_dp_geostatic", **footing(stable=True, n_steps=100, geostatic=True))
    save("terzaghi", **terzaghi())
    save("indentation3d", **indentation())
    save("jacobian_bar_j2", **jacobian_bar_j2())
    P, Q, hist = triaxial_dp()
    save("triaxial_dp", P=P, Q=Q, trial=hist)
    ax, Qn, vol = triaxial_norsand(n_steps=100)
    save("triaxial_norsand", axial=ax, Q=Qn, vol=vol)
