"""Batched inverse analysis: many independent 2D solid instances packed into one
background grid and stepped together by one engine.

Each instance is a soil block of its own size (nx x ny cells, PPD^2 particles
per cell) under ramped self-weight, with roller side walls, a fixed base and a
per-particle Young's modulus.  The blocks sit on shelves in one grid with GAP
empty cells between neighbours.  A particle's cpGIMP support reaches at most
one node beyond its cell and the Jacobian couples nodes at most two apart, so
with four empty cells no node, residual entry or matrix row is shared by two
instances: the batch is one block-diagonal system.  One cell sort, one
assembly launch, one Krylov solve, one G2P and one adjoint serve all
instances, which is what amortises the launch latency of small problems.  The
losses of the instances add, so the adjoint of their sum gives every
instance's gradient at once.

The multigrid preconditioner's coarse levels do mix neighbouring instances;
that changes the preconditioner only, not the solution.  All instances share
the grid's lp clipping box (mpm/gimp.py:449-459), which only acts on stretched
particles at the outer edge of the grid.

The workload follows the batched inverse-analysis configuration: cell counts
drawn uniformly (seeded) between 32x32 and 128x64, log Young's modulus a
Gaussian random field (mean ln 1e7, standard deviation 0.3, correlation length
0.5 m) and target displacements produced by a second field.
"""
import numpy as np
import torch

from .solvers.quasi_static_solver_2d import quasi_static_solver_2d
from .mpm.mpm_utils import init_particles_rectangle_2d

GAP = 4   # empty cells between instances
PAD = 2   # empty cells around the packed region


def instance_sizes(n, seed=0, nx_range=(32, 128), ny_range=(32, 64)):
    """(nx, ny) cell counts of n instances, uniform integers in the ranges."""
    rng = np.random.default_rng(seed)
    nx = rng.integers(nx_range[0], nx_range[1] + 1, size=n)
    ny = rng.integers(ny_range[0], ny_range[1] + 1, size=n)
    return [(int(a), int(b)) for a, b in zip(nx, ny)]


def gaussian_random_field(nx, ny, PPD, dx, corr_len, std, seed):
    """Stationary Gaussian field on the particle lattice of an nx x ny-cell block
    by Fourier filtering of white noise: covariance std^2 exp(-r^2 / corr_len^2),
    whose spectral density is proportional to exp(-|k|^2 corr_len^2 / 4).
    Returned in the particle order of init_particles_rectangle_2d
    (x cell, y cell, px, py).  The empirical mean is removed and the standard
    deviation normalised to std."""
    rng = np.random.default_rng(seed)
    mx, my = nx * PPD, ny * PPD
    h = dx / PPD
    # pad to twice the size so the periodic wrap-around does not correlate edges
    Mx, My = 2 * mx, 2 * my
    w = rng.standard_normal((Mx, My))
    kx = 2.0 * np.pi * np.fft.fftfreq(Mx, d=h)
    ky = 2.0 * np.pi * np.fft.fftfreq(My, d=h)
    k2 = kx[:, None] ** 2 + ky[None, :] ** 2
    f = np.fft.ifft2(np.fft.fft2(w) * np.sqrt(np.exp(-k2 * corr_len ** 2 / 4.0))).real[:mx, :my]
    f = (f - f.mean()) / (f.std() + 1e-300) * std
    # lattice (ix, iy) with ix = cell_x * PPD + px, iy = cell_y * PPD + py
    i, j, px, py = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(PPD), np.arange(PPD), indexing="ij")
    return f[(i * PPD + px).ravel(), (j * PPD + py).ravel()]


def shelf_pack(sizes, gap=GAP):
    """Cell offsets (ox, oy) of each block: tallest first, shelves of a common
    width chosen to make the packed region roughly square."""
    order = sorted(range(len(sizes)), key=lambda q: (-sizes[q][1], -sizes[q][0]))
    area = sum((a + gap) * (b + gap) for a, b in sizes)
    width = max(max(a for a, _ in sizes) + gap, int(np.ceil(np.sqrt(area * 1.1))))
    off = [None] * len(sizes)
    x = y = shelf_h = 0
    for q in order:
        a, b = sizes[q]
        if x > 0 and x + a > width:
            y += shelf_h + gap
            x = shelf_h = 0
        off[q] = (x, y)
        x += a + gap
        shelf_h = max(shelf_h, b)
    return off, width, y + shelf_h


class BatchedBlocks:
    """n_inst self-weight blocks in one 2D solid solver (see module docstring).

    instance(q) gives the particle slice of block q; E fields are per particle."""

    def __init__(self, sizes, dx=0.05, PPD=2, rho=2000.0, gravity=9.81, nu=0.3, material="Hencky elasticity",
                 logE=None, n_iter=20, tol=1e-6, precision="fp64", device=None, gap=GAP):
        self.sizes = list(sizes)
        self.dx, self.PPD = dx, PPD
        off, width, height = shelf_pack(self.sizes, gap)
        self.offsets = [(ox + PAD, oy + PAD) for ox, oy in off]
        n_grid_x, n_grid_y = width + 2 * PAD, height + 2 * PAD
        xs, self.slices = [], []
        start = 0
        for (nx, ny), (ox, oy) in zip(self.sizes, self.offsets):
            n = nx * ny * PPD * PPD
            xs.append(init_particles_rectangle_2d(ox * dx, oy * dx, (ox + nx) * dx, (oy + ny) * dx, dx, n_grid_x,
                                                  n_grid_y, PPD, n))
            self.slices.append(slice(start, start + n))
            start += n
        x = np.concatenate(xs)
        self.n_particles = x.shape[0]
        grid = dict(n_grid_x=n_grid_x, n_grid_y=n_grid_y, max_x=n_grid_x * dx, dx=dx, start_x=PAD * dx,
                    end_x=(n_grid_x - PAD) * dx, start_y=PAD * dx, end_y=(n_grid_y - PAD) * dx,
                    domain_min_x=PAD * dx, domain_max_x=(n_grid_x - PAD) * dx, domain_min_y=PAD * dx,
                    domain_max_y=(n_grid_y - PAD) * dx)
        parts = dict(n_particles=self.n_particles, PPD=PPD, p_vol=(dx / PPD) ** 2, p_rho=rho)
        it = dict(n_iter=n_iter, tol=tol, solver_name="warp")
        E0 = 1e7
        mat = dict(youngs_modulus=E0, poisson_ratio=nu, material_name=material)
        if logE is not None:
            mat["youngs_modulus_field"] = np.exp(np.asarray(logE, dtype=np.float64))
        load = dict(gravity_mag=gravity, traction_value_x=0.0, traction_value_y=0.0, point_load_value_x=0.0,
                    point_load_value_y=0.0)
        self.grid = grid
        self.solver = quasi_static_solver_2d(grid, parts, it, mat, load, precision=precision, device=device,
                                             x_particles=x)
        b = torch.as_tensor(self.boundary_flags(), device=self.solver.x_particles.device)
        self.solver.dofStruct.boundary_flag_array[:] = b

    def boundary_flags(self):
        """Field-major Dirichlet flags: per block, rollers on its two side node
        columns (x fixed) and a fixed base node row (x and y fixed)."""
        nx1, ny1 = self.grid["n_grid_x"] + 1, self.grid["n_grid_y"] + 1
        nn = nx1 * ny1
        b = np.zeros(2 * nn, dtype=bool)
        for (nx, ny), (ox, oy) in zip(self.sizes, self.offsets):
            iy = np.arange(oy, oy + ny + 1)
            for ix in (ox, ox + nx):
                b[ix + iy * nx1] = True
            ix = np.arange(ox, ox + nx + 1)
            b[ix + oy * nx1] = True
            b[ix + oy * nx1 + nn] = True
        return b

    def instance(self, q):
        return self.slices[q]

    def reset_state(self):
        """Back to the undeformed start (positions, F, b, lp, stress)."""
        e = self.solver.engine
        e.x.copy_(e.x0)
        ident = torch.tensor([[1.0 + 1e-7, 0, 0], [0, 1.0 - 1e-6, 0], [0, 0, 1.0]], dtype=torch.float64,
                             device=e.device)
        for t in (e.F_old, e.F_new, e.b_old, e.b_new):
            t[:] = ident
        e.lp.fill_(self.solver.GIMP_lp_initial)
        e.sigma.zero_()

    def displacement(self):
        s = self.solver
        return s.x_particles - s.x0


def random_fields(sizes, seed, dx=0.05, PPD=2, mean=np.log(1e7), std=0.3, corr_len=0.5):
    """Concatenated per-particle log E of every block (block q uses seed + q)."""
    return np.concatenate([mean + gaussian_random_field(nx, ny, PPD, dx, corr_len, std, seed + q)
                           for q, (nx, ny) in enumerate(sizes)])
