"""Implicit cpGIMP load step, CPU oracle (NumPy/SciPy FP64).

Restates the reference's per-particle residual kernels and solver loops:

  residual, 2D solid (Hencky / J2)   mpm/mpm_utils.py:416-780
  residual, 2D u-p (neo-Hookean)     mpm/mpm_utils.py:782-1017
  residual, 3D u-p (neo-Hookean,
            penalty footing)          mpm/mpm_utils.py:1020-1294
  P2G activation / pressure BCs /
  consistent-mass projection         mpm/mpm_utils.py:83-414
  Jacobian masks and identity rows   solvers/sparse_differentiation.py:213-401,
                                     mpm/mpm_utils.py:1299-1341
  Newton loop ('scipy' path)         solvers/quasi_static_solver_2d.py:151-231
  G2P + lp update                    mpm/mpm_utils.py:1351-1590, mpm/gimp.py:428-507

Extensions beyond the reference (documented, same residual structure):
Neo-Hookean and small-strain linear elasticity and Drucker-Prager/NorSand in
the 2D solid solver, a 2D restatement of the 3D penalty footing, linear
elasticity and Drucker-Prager in the u-p solvers, and per-particle Young's
modulus.  The Jacobian K = -dR/du is built element by element by complex-step
differentiation of each particle's residual with respect to its local nodal
unknowns (exact to round-off), replacing Warp's coloured reverse-mode sweeps.

Test infrastructure only: see the package docstring.
"""
import numpy as np
import scipy.sparse as sp
from scipy.sparse.linalg import spsolve

from . import gimp as G
from .eig import eigh3, from_principal
from . import materials as MT
from . import native

CS_H = 1e-30  # complex-step size


# ------------------------------------------------------------------ seeding
def init_particles_rectangle_2d(start_x, start_y, end_x, end_y, dx, n_grid_x, n_grid_y, PPD, n_particles):
    """mpm/mpm_utils.py:12-29 (same order: x cell, y cell, then px, py)."""
    out = np.zeros((n_particles, 2))
    pid = 0
    for i in range(n_grid_x):
        for j in range(n_grid_y):
            cx, cy = (i + 0.5) * dx, (j + 0.5) * dx
            if start_x < cx < end_x and start_y < cy < end_y:
                for px in range(PPD):
                    for py in range(PPD):
                        out[pid] = np.array([i * dx, j * dx]) + np.array([(0.5 + px) * dx / PPD, (0.5 + py) * dx / PPD])
                        pid += 1
    return out


def init_particles_rectangle_3d(start_x, start_y, start_z, end_x, end_y, end_z, dx, n_grid_x, n_grid_y, n_grid_z, PPD, n_particles):
    """mpm/mpm_utils.py:31-51."""
    out = np.zeros((n_particles, 3))
    pid = 0
    for i in range(n_grid_x):
        for j in range(n_grid_y):
            for k in range(n_grid_z):
                cx, cy, cz = (i + 0.5) * dx, (j + 0.5) * dx, (k + 0.5) * dx
                if start_x < cx < end_x and start_y < cy < end_y and start_z < cz < end_z:
                    for px in range(PPD):
                        for py in range(PPD):
                            for pz in range(PPD):
                                out[pid] = np.array([i * dx, j * dx, k * dx]) + np.array(
                                    [(0.5 + px) * dx / PPD, (0.5 + py) * dx / PPD, (0.5 + pz) * dx / PPD])
                                pid += 1
    return out


def perturbed_identity(n):
    """Initial F and b, mpm/mpm_utils.py:53-74: diag(1+1e-7, 1-1e-6, 1)."""
    M = np.zeros((n, 3, 3))
    M[:, 0, 0] = 1.0 + 1e-7
    M[:, 1, 1] = 1.0 - 1e-6
    M[:, 2, 2] = 1.0
    return M


# ------------------------------------------------------------------ helpers
def det3(A):
    return (A[:, 0, 0] * (A[:, 1, 1] * A[:, 2, 2] - A[:, 1, 2] * A[:, 2, 1])
            - A[:, 0, 1] * (A[:, 1, 0] * A[:, 2, 2] - A[:, 1, 2] * A[:, 2, 0])
            + A[:, 0, 2] * (A[:, 1, 0] * A[:, 2, 1] - A[:, 1, 1] * A[:, 2, 0]))


def inv2(A):
    d = A[:, 0, 0] * A[:, 1, 1] - A[:, 0, 1] * A[:, 1, 0]
    out = np.empty_like(A)
    out[:, 0, 0] = A[:, 1, 1] / d
    out[:, 1, 1] = A[:, 0, 0] / d
    out[:, 0, 1] = -A[:, 0, 1] / d
    out[:, 1, 0] = -A[:, 1, 0] / d
    return out


def embed3(A2):
    A = np.zeros((A2.shape[0], 3, 3), dtype=A2.dtype)
    A[:, :2, :2] = A2
    A[:, 2, 2] = 1.0
    return A


def mm(A, B):
    return np.einsum("nij,njk->nik", A, B)


def mv(A, v):
    return np.einsum("nij,nj->ni", A, v)


def lame(E, nu):
    return E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)), E / (2.0 * (1.0 + nu))


# ------------------------------------------------------------------ constitutive dispatch
SPECTRAL_MODELS = ("Hencky elasticity", "J2", "Drucker-Prager", "NorSand")


def spectral_update(b_trial, J, mat, lam, mu, pi_old, pi_new):
    """Trial b -> Kirchhoff stress via principal log strains.

    Restates mpm/mpm_utils.py:521-560 (eig3, e = 0.5 log max(lambda, 1e-8),
    return map, tau = sum tau_A n_A n_A^T, b_new = sum exp(2 e_A) n_A n_A^T).
    Returns (tau[N,3,3], b_new[N,3,3], pi_new).
    """
    name = mat["material_name"]
    lamb, V = eigh3(b_trial)
    lr = np.real(lamb)
    e_tr = 0.5 * np.log(np.where(lr > 1e-8, lamb, 1e-8))
    pi_out = pi_new
    if name == "Hencky elasticity":
        e = e_tr
        tau_p = MT.kirchhoff_hencky(e, lam[:, None], mu[:, None])
    elif name == "J2":
        e = MT.return_map_j2(e_tr, lam[:, None], mu[:, None], mat["kappa"])
        tau_p = MT.kirchhoff_hencky(e, lam[:, None], mu[:, None])
    elif name == "Drucker-Prager":
        e = MT.return_map_dp(e_tr, lam[:, None], mu[:, None], mat["friction_angle"], mat["dilation_angle"],
                             mat["cohesion"], mat.get("shape_factor", 0.0),
                             tension_cutoff=mat.get("tension_cutoff", True))
        tau_p = MT.kirchhoff_hencky(e, lam[:, None], mu[:, None])
    elif name == "NorSand":
        prm = norsand_params(mat)
        eps_v_total = np.log(J) + prm["eps_v0"]
        e, pi_out = MT.return_map_norsand(e_tr, eps_v_total, pi_old, pi_new, prm)
        tau_p = MT.kirchhoff_norsand(e, prm)
    else:
        raise ValueError(f"Unimplemented material model: {name}")
    tau = from_principal(tau_p, V)
    b_new = from_principal(np.exp(2.0 * e), V)
    return tau, b_new, pi_out


def norsand_params(mat):
    return {k: mat[k] for k in ("kappa", "tilde_lambda", "M", "N", "beta", "vc0", "p0", "v0", "h")} | {
        "mu": mat["shear_modulus"], "eps_v0": mat.get("initial_volumetric_strain", 0.0)}


def cauchy_neohookean_2d(F_new, J, lam, mu):
    """mpm/mpm_utils.py:915 (2D u-p form)."""
    I = np.eye(3)
    return (mu / J)[:, None, None] * (mm(F_new, np.swapaxes(F_new, 1, 2)) - I) + (lam / J * np.log(J))[:, None, None] * I


def cauchy_neohookean_3d(F_new, J, lam, mu):
    """mpm/mpm_utils.py:1205-1208 (PK1 form)."""
    Finv = np.linalg.inv(F_new)
    FinvT = np.swapaxes(Finv, 1, 2)
    P = mu[:, None, None] * (F_new - FinvT) + (lam * np.log(J))[:, None, None] * FinvT
    return (1.0 / J)[:, None, None] * mm(P, np.swapaxes(F_new, 1, 2))


def cauchy_linear(F_new, lam, mu):
    """Small-strain linear elasticity on eps = sym(F) - I (extension)."""
    I = np.eye(3)
    eps = 0.5 * (F_new + np.swapaxes(F_new, 1, 2)) - I
    tr = np.trace(eps, axis1=1, axis2=2)
    return (lam * tr)[:, None, None] * I + 2.0 * mu[:, None, None] * eps


# ------------------------------------------------------------------ the engine
class OracleEngine:
    """One implicit cpGIMP problem (2D solid, 2D u-p or 3D u-p), CPU FP64.

    kind: 'solid2d' | 'coupled2d' | 'coupled3d'.
    grid: dict with n_grid (tuple), h (cell sizes used by the shape functions),
          h_nodes (cell sizes used for nodal positions), domain_min/max tuples.
    """

    def __init__(self, kind, grid, x, p_vol, p_rho, PPD, mat, load, lp0, n_iter=10, tol=1e-8, dt=0.0,
                 phi_initial=0.0, mobility=0.0, E_field=None, act_thresh=None, mobility_law="constant",
                 p2g_projection="consistent"):
        self.kind = kind
        self.threads = 1  # host threads for the tangent's complex-step passes (timing runs raise it)
        # the compiled per-particle residual and tangent (oracle/native.py) for
        # the cases it covers; off by default, so the tests check the NumPy path
        self.use_native = False
        self.D = 2 if kind in ("solid2d", "coupled2d") else 3
        self.nf = {"solid2d": 2, "coupled2d": 3, "coupled3d": 4}[kind]
        self.grid = dict(grid)
        self.n_grid = tuple(grid["n_grid"])
        self.n_nodes = int(np.prod([n + 1 for n in self.n_grid]))
        self.ndof = self.nf * self.n_nodes
        self.x = np.array(x, dtype=np.float64)
        self.x0 = self.x.copy()
        self.N = self.x.shape[0]
        self.p_vol, self.p_rho, self.PPD = p_vol, p_rho, PPD
        self.p_mass = p_vol * p_rho
        self.mat = dict(mat)
        self.load = dict(load)
        self.lp0 = lp0
        self.n_iter, self.tol, self.dt = n_iter, tol, dt
        self.phi_initial, self.mobility = phi_initial, mobility
        E = mat["youngs_modulus"] if E_field is None else E_field
        self.E = np.broadcast_to(np.asarray(E, dtype=np.float64), (self.N,)).copy()
        self.nu = mat["poisson_ratio"]
        self.act_thresh = act_thresh
        self.mobility_law = mobility_law
        self.p2g_projection = p2g_projection
        self.F_new = perturbed_identity(self.N)
        self.F_old = perturbed_identity(self.N)
        self.b_new = perturbed_identity(self.N)
        self.b_old = perturbed_identity(self.N)
        self.sigma = np.zeros((self.N, 3, 3))
        self.lp = np.full((self.N, self.D), lp0)
        self.pressure = np.zeros(self.N)
        self.ext_flag = np.zeros(self.N, dtype=bool)
        self.trac_flag = np.zeros(self.N, dtype=bool)
        self.pbc_flag = np.zeros(self.N, dtype=bool)
        pi0 = mat.get("pi_initial", 0.0)
        self.pi_old = np.full(self.N, pi0)
        self.pi_new = np.full(self.N, pi0)
        self.boundary = np.zeros(self.ndof, dtype=bool)
        self.active = np.zeros(self.ndof, dtype=bool)
        self.u_old = np.zeros(self.ndof)
        self.u_new = np.zeros(self.ndof)
        self.force = 0.0
        self.iters = []
        self.res_norms = []
        self.last_K = None
        self.last_R = None

    # ---------------- geometry
    def shape(self):
        h = self.grid["h"]
        inv_h = tuple(1.0 / v for v in h)
        lower, span, w, gw, wavg = G.gimp(self.x, self.lp, h, inv_h)
        W, Gr, Wa = G.nodal_weights(w, gw, wavg)
        ids, valid = G.node_ids(lower, self.n_grid)
        return lower, span, W, Gr, Wa, ids, valid

    def dof(self, ids, f):
        return ids + f * self.n_nodes

    # ---------------- P2G (activation, pressure BCs, consistent mass)
    def p2g(self):
        lower, span, W, Gr, Wa, ids, valid = self.shape()
        tab = G.node_tables(self.D)
        self.active[:] = False
        if self.kind == "solid2d":
            # mpm/mpm_utils.py:115-136: span nodes, no weight threshold
            for a, idx in enumerate(tab):
                m = valid[:, a] & np.all([idx[k] < span[:, k] for k in range(self.D)], axis=0)
                for f in range(self.nf):
                    self.active[self.dof(ids[m, a], f)] = True
            return
        thr = 1e-6 if self.kind == "coupled2d" else 1e-7
        if self.act_thresh is not None:
            thr = self.act_thresh
        for a, idx in enumerate(tab):
            if self.kind == "coupled2d":
                in_span = np.all([idx[k] < span[:, k] for k in range(self.D)], axis=0)
            else:
                in_span = np.ones(self.N, dtype=bool)  # 3D loops over all 27 (mpm_utils.py:327)
            m = valid[:, a] & in_span & (np.real(W[:, a]) > thr)
            for f in range(self.nf):
                self.active[self.dof(ids[m, a], f)] = True
        # pressure Dirichlet nodes above flagged particles (mpm_utils.py:225-235, 349-352)
        hn = self.grid["h_nodes"]
        pf = self.nf - 1
        for a, idx in enumerate(tab):
            if self.kind == "coupled2d":
                in_span = np.all([idx[k] < span[:, k] for k in range(self.D)], axis=0)
            else:
                in_span = np.ones(self.N, dtype=bool)
            vert = self.D - 1
            node_v = (lower[:, vert] + idx[vert]).astype(np.float64) * hn[vert]
            m = valid[:, a] & in_span & self.pbc_flag & (node_v >= self.x[:, vert])
            self.boundary[self.dof(ids[m, a], pf)] = True
        # consistent-mass projection (mpm_utils.py:237-257, 354-383); exact solve
        rows = np.repeat(ids, ids.shape[1], axis=1).ravel()
        cols = np.tile(ids, (1, ids.shape[1])).ravel()
        ok = (np.repeat(valid, ids.shape[1], axis=1) & np.tile(valid, (1, ids.shape[1]))).ravel()
        vals = (W[:, :, None] * W[:, None, :] * self.p_mass).ravel()
        M = sp.coo_matrix((vals[ok], (rows[ok], cols[ok])), shape=(self.n_nodes, self.n_nodes)).tocsr()
        rhs = np.zeros(self.n_nodes)
        wsum = np.where(valid, W, 0.0).sum(1)  # literal: sum_b W_a W_b m p (mpm_utils.py:254)
        np.add.at(rhs, ids[valid], (W * wsum[:, None] * self.p_mass * self.pressure[:, None])[valid])
        diag = M.diagonal()
        zero = diag == 0.0
        M = M + sp.diags(zero.astype(np.float64))  # untouched nodes: p_hat = 0
        if self.p2g_projection == "lumped":
            # P2G_solver_lumped (large_consolidation_cpGIMP_everything_in_one_script.py:292-310):
            # p_i = sum N m p / sum N m, the lumped mass being the row sum of M
            msum = np.asarray(M.sum(axis=1)).ravel() - zero  # untouched rows: the unit diagonal added above
            xp = np.where(msum != 0.0, rhs / np.where(msum != 0.0, msum, 1.0), 0.0)
        else:
            xp = spsolve(M.tocsc(), rhs)
        pdof = np.arange(self.n_nodes) + pf * self.n_nodes
        sel = ~self.boundary[pdof]
        if self.kind == "coupled3d":
            sel &= self.active[pdof]  # mpm_utils.py:401-414
        self.u_old[pdof[sel]] = xp[sel]
        self.u_new[pdof[sel]] = xp[sel]
        self.mass_matrix = M
        self.mass_rhs = rhs
        self.p_hat = xp

    # ---------------- local residuals
    def local(self, Uloc_new, Uloc_old, geo, step, n_steps, want_aux=False):
        """Per-particle residual contributions r[N, A, nf] for local nodal values."""
        lower, span, W, Gr, Wa, ids, valid = geo
        D = self.D
        dtype = Uloc_new.dtype
        lam, mu = lame(self.E, self.nu)
        ramp = (step + 1.0) / n_steps
        dU = Uloc_new[:, :, :D] - Uloc_old[:, :, :D]
        Hd = np.einsum("nak,nal->nkl", Gr, dU)
        Finc = np.eye(D)[None] + Hd
        if D == 2:
            Finv = inv2(Finc)
            Finc3 = embed3(Finc)
        else:
            Finv = np.linalg.inv(Finc)
            Finc3 = Finc
        F_new = mm(Finc3, self.F_old.astype(dtype))
        J = det3(F_new)
        J_old = det3(self.F_old)
        name = self.mat["material_name"]
        pi_new = self.pi_new
        if name in SPECTRAL_MODELS:
            b_tr = mm(mm(Finc3, self.b_old), np.swapaxes(Finc3, 1, 2))
            tau, b_new, pi_new = spectral_update(b_tr, J, self.mat, lam, mu, self.pi_old, self.pi_new)
            sig3 = tau / J[:, None, None]
        else:
            b_new = mm(mm(Finc3, self.b_old), np.swapaxes(Finc3, 1, 2))
            if name == "Neo-Hookean":
                sig3 = cauchy_neohookean_3d(F_new, J, lam, mu) if D == 3 else cauchy_neohookean_2d(F_new, J, lam, mu)
            elif name == "Linear elasticity":
                sig3 = cauchy_linear(F_new, lam, mu)
            else:
                raise ValueError(f"Unimplemented material model: {name}")
        sig = sig3[:, :D, :D]
        V_new = self.p_vol * J
        g = np.zeros(D)
        # gravity_ramp False (extension): full gravity from the first load step
        g[D - 1] = -self.load.get("gravity_mag", 0.0) * (ramp if self.load.get("gravity_ramp", True) else 1.0)
        Ggrad = np.einsum("nkl,nal->nak", Finv, Gr)  # incr_F_inv @ weight_GRAD
        r = np.zeros(Uloc_new.shape[:2] + (self.nf,), dtype=np.result_type(dtype, sig))
        fext = np.zeros((self.N, D))
        pl = [self.load.get(k, 0.0) for k in ("point_load_value_x", "point_load_value_y", "point_load_value_z")[:D]]
        fext[self.ext_flag] = np.array(pl) * ramp
        force = 0.0
        if self.kind == "solid2d":
            rho_new = self.p_rho / J
            r[:, :, :2] = (-np.einsum("nai,nij->naj", Ggrad, sig) + (W * rho_new[:, None])[:, :, None] * g) * V_new[:, None, None] \
                + W[:, :, None] * fext[:, None, :]
            pen, force = self.penalty(W, dU, lam, mu, step)
            if pen is not None:
                r[:, :, D - 1] += pen
        else:
            pf = self.nf - 1
            p_new = Uloc_new[:, :, pf]
            p_old = Uloc_old[:, :, pf]
            pbar = (W * p_new).sum(1)
            pbar_old = (W * p_old).sum(1)
            pavg = (Wa * p_new).sum(1)
            pavg_old = (Wa * p_old).sum(1)
            if D == 2:
                gradp = np.einsum("nak,na->nk", Ggrad, p_new)  # mpm_utils.py:950 (spatial gradient)
            else:
                gradp = np.einsum("nak,na->nk", Gr, p_new)  # mpm_utils.py:1194 (reference gradient)
            phi_s0 = 1.0 - self.phi_initial
            n_f = 1.0 - phi_s0 / J
            rho_mix = n_f * 1.0 + (1.0 - n_f) * self.p_rho
            tauppp = 0.5 / mu
            ftr = np.zeros((self.N, D))
            tv = [self.load.get(k, 0.0) for k in ("traction_value_x", "traction_value_y", "traction_value_z")[:D]]
            hh = self.grid["h"]
            ftr[self.trac_flag] = np.array([tv[k] * hh[k] / self.PPD for k in range(D)])
            eff = sig - pbar[:, None, None] * np.eye(D)
            r[:, :, :D] = (-np.einsum("nai,nij->naj", Ggrad, eff) + (W * rho_mix[:, None])[:, :, None] * g) * V_new[:, None, None]
            if D == 2:
                # point load and traction enter only the 2D momentum residual (mpm_utils.py:994);
                # the 3D kernel computes them but never adds them (mpm_utils.py:1271)
                r[:, :, :D] += W[:, :, None] * fext[:, None, :] + W[:, :, None] * ftr[:, None, :]
            else:
                pen, force = self.penalty(W, dU, lam, mu, step)
                if pen is not None:
                    r[:, :, D - 1] += pen
            mob = self.mobility
            if self.mobility_law == "Uzuoka-Borja":
                # large_consolidation_cpGIMP_everything_in_one_script.py:330-338 (Eq. 86 of Uzuoka & Borja)
                mob = mob * ((2.0 * mu + lam) * J) / (mu * (1.0 + 1.0 / J ** 2) + (1.0 - np.log(J)) * lam / J ** 2)
                mob = mob[:, None]
            r[:, :, pf] =(W * (np.log(J) - np.log(J_old))[:, None]
                           + np.einsum("nak,nk->na", Ggrad, mob * gradp) * self.dt) * V_new[:, None]
            r[:, :, pf] += (tauppp[:, None] * (W - Wa) * (pbar - pavg - (pbar_old - pavg_old))[:, None]) * V_new[:, None]
        if want_aux:
            return r, dict(F_new=F_new, b_new=b_new, sigma=sig3, pi_new=pi_new, force=force)
        return r

    def penalty(self, W, dU, lam, mu, step):
        """Penalty footing: mpm/mpm_utils.py:1234-1248 (3D); the 2D solver restates it with y vertical."""
        ld = self.load
        if "penalty_factor" not in ld:
            return None, 0.0
        D = self.D
        v = D - 1
        h = self.grid["h"]
        area = h[0] / self.PPD if D == 2 else (h[0] / self.PPD) * (h[1] / self.PPD)
        kpen = self.E * ld["penalty_factor"] * area
        height = ld["footing_initial_height"] + (step + 1.0) * ld["footing_incr_disp"]
        xp = self.x
        sel = (xp[:, v] >= height) & (xp[:, 0] > ld["footing_region_min_x"]) & (xp[:, 0] < ld["footing_region_max_x"])
        if D == 3:
            sel &= (xp[:, 1] > ld["footing_region_min_y"]) & (xp[:, 1] < ld["footing_region_max_y"])
        du = (W * dU[:, :, v]).sum(1)
        pen_res = -(height - (xp[:, v] + du)) * kpen
        if ld.get("footing_penalty_stable", False):
            pen_res = -pen_res  # attractive spring to the footing height (extension)
        pen_res = np.where(sel, pen_res, 0.0)
        return pen_res[:, None] * W, np.real(-pen_res[sel]).sum()

    # ---------------- global assembly
    def gather(self, vec, ids, valid):
        out = np.zeros(ids.shape + (self.nf,))
        for f in range(self.nf):
            v = vec[np.where(valid, ids, 0) + f * self.n_nodes]
            out[:, :, f] = np.where(valid, v, 0.0)
        return out

    def assemble(self, step, n_steps, want_K=True):
        geo = self.shape()
        lower, span, W, Gr, Wa, ids, valid = geo
        Un = self.gather(self.u_new, ids, valid)
        Uo = self.gather(self.u_old, ids, valid)
        nat = self.use_native and native.supports(self)
        if nat:
            r, K_loc, aux = native.solid2d_local(self, geo, Un, Uo, step, n_steps, want_K)
        else:
            r, aux = self.local(Un, Uo, geo, step, n_steps, want_aux=True)
        free = self.active & ~self.boundary
        A = ids.shape[1]
        R = np.zeros(self.ndof)
        dofs = np.stack([ids + f * self.n_nodes for f in range(self.nf)], 2)  # [N, A, nf]
        okd = valid[:, :, None] & free[np.where(valid[:, :, None], dofs, 0)]
        np.add.at(R, dofs[okd], np.real(r)[okd])
        K = None
        if want_K and nat:
            # the same entries as the complex-step passes below: row (a, f) and
            # column (b, g) of every particle where both DOFs are free
            rr, cc, vv = native.triplets(self, dofs, okd, K_loc)
            rows, cols, vals = [rr], [cc], [vv]
        elif want_K:
            def column(bg):
                # complex-step pass for local column (b, g): K = -dR/du
                b, g = bg
                Up = Un.astype(np.complex128)
                Up[:, b, g] += 1j * CS_H
                rp = self.local(Up, Uo, geo, step, n_steps)
                dcol = -np.imag(rp) / CS_H
                colok = valid[:, b] & free[np.where(valid[:, b], dofs[:, b, g], 0)]
                m = okd & colok[:, None, None]
                return (dofs[m], np.broadcast_to(dofs[:, b, g][:, None, None], dofs.shape)[m], dcol[m])

            passes = [(b, g) for b in range(A) for g in range(self.nf)]
            if self.threads > 1:
                # the passes are independent NumPy work (the GIL is released in
                # it); results are kept in pass order, so K is the same
                from concurrent.futures import ThreadPoolExecutor
                with ThreadPoolExecutor(self.threads) as ex:
                    parts = list(ex.map(column, passes))
            else:
                parts = [column(bg) for bg in passes]
            rows = [r for r, _, _ in parts]
            cols = [c for _, c, _ in parts]
            vals = [v for _, _, v in parts]
        if want_K:
            nf_rows = np.where(~free)[0]
            rows.append(nf_rows)
            cols.append(nf_rows)
            vals.append(np.ones(nf_rows.size))
            K = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                              shape=(self.ndof, self.ndof)).tocsr()
        return R, K, aux

    # ---------------- step
    def newton(self, step, n_steps):
        its = 0
        for it in range(self.n_iter):
            R, K, aux = self.assemble(step, n_steps)
            self.F_new, self.b_new, self.sigma = aux["F_new"].real, aux["b_new"].real, aux["sigma"].real
            self.pi_new = np.real(aux["pi_new"]) if np.ndim(aux["pi_new"]) else self.pi_new
            self.force = aux["force"]
            self.last_K, self.last_R = K, R
            delta = spsolve(K.tocsc(), R)
            self.u_new += delta
            its += 1
            nrm = np.linalg.norm(R)
            self.res_norms.append(nrm)
            if nrm < self.tol:
                break
        self.iters.append(its)

    def g2p(self):
        geo = self.shape()
        lower, span, W, Gr, Wa, ids, valid = geo
        Un = self.gather(self.u_new, ids, valid)
        Uo = self.gather(self.u_old, ids, valid)
        du = np.einsum("na,naf->nf", W, Un[:, :, :self.D] - Uo[:, :, :self.D])
        self.F_old = self.F_new.copy()
        self.b_old = self.b_new.copy()
        self.pi_old = self.pi_new.copy()
        self.x = self.x + du
        if self.kind != "solid2d":
            self.pressure = np.einsum("na,na->n", W, Un[:, :, self.nf - 1])
        self.lp = G.update_lp(self.F_new, self.x, self.lp0, self.grid["domain_min"], self.grid["domain_max"])

    def advance_one_step(self, step, n_steps, set_boundary=None):
        """One load step: reset, [BCs], P2G, Newton, G2P, lp update."""
        self.u_old[:] = 0.0
        self.u_new[:] = 0.0
        if self.kind != "solid2d":
            self.boundary[:] = False
            if set_boundary is not None:
                set_boundary(self.boundary)
        self.p2g()
        self.newton(step, n_steps)
        self.g2p()
