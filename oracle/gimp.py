"""cpGIMP shape functions (oracle, NumPy, complex-step capable).

Restates mpm/gimp.py:25-425 (standard and cell-averaged cpGIMP weights, after
Coombs et al. section 2.4.2) and mpm/gimp.py:428-507 (lp update after
Charlton et al. 2017, Eqs. 38-39).  All functions are vectorised over particles
and accept complex arrays so that complex-step derivatives propagate.
"""
import numpy as np


def rabs(z):
    """|z| continued analytically (sign taken from the real part)."""
    return np.where(np.real(z) < 0, -z, z)


def rsign(z):
    """wp.sign on the real part: -1 for negative, +1 otherwise."""
    return np.where(np.real(z) < 0, -1.0, 1.0)


def cell_index(coord, inv_d):
    """int(coord*inv_d + 1e-8) with C truncation (mpm/gimp.py:34-36)."""
    return np.trunc(np.real(coord) * inv_d + 1e-8).astype(np.int64)


def gimp_axis(xp, lp, d, inv_d):
    """One axis of the cpGIMP weights for arrays of particle coordinates.

    Returns (lower, span, w, gw, wavg) with w, gw, wavg of shape [..., 3]:
    node k of the particle sits at (lower + k)*d.  Follows
    mpm/gimp.py:33-108 (standard) and mpm/gimp.py:156-189 (averaged).
    """
    lower = cell_index(xp - lp, inv_d)
    upper = cell_index(xp + lp, inv_d)
    base = cell_index(xp, inv_d)
    fx = xp * inv_d - base.astype(np.float64)
    same = upper == lower
    dt = np.result_type(xp, lp, np.float64)
    shape = np.shape(xp) + (3,)
    w = np.zeros(shape, dtype=dt)
    gw = np.zeros(shape, dtype=dt)
    wavg = np.zeros(shape, dtype=dt)

    lowf = lower.astype(np.float64)
    x0 = lowf * d
    x1 = (lowf + 1.0) * d
    x2 = (lowf + 2.0) * d
    a0 = rabs(xp - x0)
    a2 = rabs(xp - x2)
    with np.errstate(divide="ignore", invalid="ignore"):
        w0_3 = (d + lp - a0) ** 2 / (4.0 * d * lp)
        g0_3 = -(d + lp - a0) / (2.0 * d * lp) * (xp - x0) / a0
        w1_3 = 1.0 - ((xp - x1) ** 2 + lp ** 2) / (2.0 * d * lp)
        g1_3 = -(xp - x1) / (d * lp)
        w2_3 = (d + lp - a2) ** 2 / (4.0 * d * lp)
        g2_3 = -(d + lp - a2) / (2.0 * d * lp) * (xp - x2) / a2
        v0_3 = (d + lp - a0) / (4.0 * lp)
        v2_3 = (d + lp - a2) / (4.0 * lp)

    w[..., 0] = np.where(same, 1.0 - fx, w0_3)
    w[..., 1] = np.where(same, fx, w1_3)
    w[..., 2] = np.where(same, 0.0, w2_3)
    gw[..., 0] = np.where(same, -inv_d, g0_3)
    gw[..., 1] = np.where(same, inv_d, g1_3)
    gw[..., 2] = np.where(same, 0.0, g2_3)
    wavg[..., 0] = np.where(same, 0.5, v0_3)
    wavg[..., 1] = 0.5
    wavg[..., 2] = np.where(same, 0.0, v2_3)
    span = np.where(same, 2, 3)
    return lower, span, w, gw, wavg


def gimp(x, lp, h, inv_h):
    """Shape data for particles x[N, D] with half-widths lp[N, D].

    h / inv_h: per-axis cell sizes.  In 2D the reference uses dx for both axes
    (mpm/gimp.py:26-31); callers pass (dx, dx) there.
    Returns lower[N, D] (int), span[N, D], w[N, 3, D], gw[N, 3, D], wavg[N, 3, D].
    """
    D = x.shape[1]
    lowers, spans, ws, gws, wavgs = [], [], [], [], []
    for k in range(D):
        lo, sp, w, gw, wa = gimp_axis(x[:, k], lp[:, k], h[k], inv_h[k])
        lowers.append(lo)
        spans.append(sp)
        ws.append(w)
        gws.append(gw)
        wavgs.append(wa)
    return (np.stack(lowers, 1), np.stack(spans, 1), np.stack(ws, 2),
            np.stack(gws, 2), np.stack(wavgs, 2))


def node_tables(D):
    """Local node enumeration a -> (i, j[, k]) used everywhere in the oracle.

    a = i + 3 j (+ 9 k): the slot order of the reference's consistent-mass
    triplets (mpm/mpm_utils.py:255, 381).
    """
    if D == 2:
        return [(a % 3, a // 3) for a in range(9)]
    return [(a % 3, (a // 3) % 3, a // 9) for a in range(27)]


def nodal_weights(w, gw, wavg):
    """Tensor-product weights per local node.

    Returns W[N, A], G[N, A, D] (reference gradient weight_GRAD), Wavg[N, A].
    """
    N, _, D = w.shape
    tab = node_tables(D)
    A = len(tab)
    W = np.empty((N, A), dtype=w.dtype)
    Wa = np.empty((N, A), dtype=w.dtype)
    G = np.empty((N, A, D), dtype=w.dtype)
    for a, idx in enumerate(tab):
        W[:, a] = np.prod([w[:, idx[k], k] for k in range(D)], axis=0)
        Wa[:, a] = np.prod([wavg[:, idx[k], k] for k in range(D)], axis=0)
        for c in range(D):
            G[:, a, c] = np.prod([gw[:, idx[k], k] if k == c else w[:, idx[k], k]
                                  for k in range(D)], axis=0)
    return W, G, Wa


def node_ids(lower, n_grid):
    """Global node ids of the 3^D local nodes: ix + iy (nx+1) [+ iz (nx+1)(ny+1)].

    Also returns a validity mask for nodes inside the grid.
    """
    N, D = lower.shape
    tab = node_tables(D)
    ids = np.empty((N, len(tab)), dtype=np.int64)
    valid = np.ones((N, len(tab)), dtype=bool)
    for a, idx in enumerate(tab):
        nid = np.zeros(N, dtype=np.int64)
        stride = 1
        for k in range(D):
            c = lower[:, k] + idx[k]
            valid[:, a] &= (c >= 0) & (c <= n_grid[k])
            nid += c * stride
            stride *= n_grid[k] + 1
        ids[:, a] = nid
    return ids, valid


def update_lp(F_new, x, lp0, dmin, dmax):
    """lp = lp0 * |F column| clipped to the domain (mpm/gimp.py:428-507)."""
    D = x.shape[1]
    lp = np.empty_like(x)
    for k in range(D):
        U = np.sqrt(F_new[:, 0, k] ** 2 + F_new[:, 1, k] ** 2 + F_new[:, 2, k] ** 2)
        v = lp0 * U
        v = np.where(x[:, k] - v < dmin[k], x[:, k] - dmin[k] - 1e-6, v)
        v = np.where(x[:, k] + v > dmax[k], dmax[k] - x[:, k] - 1e-6, v)
        lp[:, k] = v
    return lp
