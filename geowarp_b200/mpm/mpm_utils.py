"""Host-side helpers with the reference's names (mpm/mpm_utils.py:12-51)."""
import numpy as np


def init_particles_rectangle_2d(start_x, start_y, end_x, end_y, dx, n_grid_x, n_grid_y, PPD, n_particles):
    """Regular PPD x PPD seeding in every cell whose centre lies strictly inside
    the box; order: x cell, y cell, then px, py (mpm/mpm_utils.py:12-29)."""
    i = np.arange(n_grid_x)
    j = np.arange(n_grid_y)
    ci = (i + 0.5) * dx
    cj = (j + 0.5) * dx
    I = i[(start_x < ci) & (ci < end_x)]
    J = j[(start_y < cj) & (cj < end_y)]
    pp = np.arange(PPD)
    # index order (i, j, px, py)
    ii, jj, px, py = np.meshgrid(I, J, pp, pp, indexing="ij")
    x = ii * dx + (0.5 + px) * dx / PPD
    y = jj * dx + (0.5 + py) * dx / PPD
    out = np.zeros((n_particles, 2))
    pts = np.stack([x.ravel(), y.ravel()], 1)
    if pts.shape[0] > n_particles:
        raise ValueError(f"box holds {pts.shape[0]} particles, more than n_particles={n_particles}")
    out[: pts.shape[0]] = pts
    return out


def init_particles_rectangle_3d(start_x, start_y, start_z, end_x, end_y, end_z, dx, n_grid_x, n_grid_y, n_grid_z,
                                PPD, n_particles):
    """3D version (mpm/mpm_utils.py:31-51): order x, y, z cell then px, py, pz."""
    ax = []
    for start, end, n in ((start_x, end_x, n_grid_x), (start_y, end_y, n_grid_y), (start_z, end_z, n_grid_z)):
        i = np.arange(n)
        c = (i + 0.5) * dx
        ax.append(i[(start < c) & (c < end)])
    pp = np.arange(PPD)
    ii, jj, kk, px, py, pz = np.meshgrid(ax[0], ax[1], ax[2], pp, pp, pp, indexing="ij")
    pts = np.stack([(ii * dx + (0.5 + px) * dx / PPD).ravel(), (jj * dx + (0.5 + py) * dx / PPD).ravel(),
                    (kk * dx + (0.5 + pz) * dx / PPD).ravel()], 1)
    out = np.zeros((n_particles, 3))
    if pts.shape[0] > n_particles:
        raise ValueError(f"box holds {pts.shape[0]} particles, more than n_particles={n_particles}")
    out[: pts.shape[0]] = pts
    return out
